// Incremental (dP) RHF G builds: the GPU form of the reference's
// EriDirectJKIncrementalState (integrals/two_electron/fock/eri_direct_jk.hpp:
// 41-135, fock/detail/direct_build.ipp:562-775).
//
// The cached density and G stay on the device.  One update:
//   1. stage the new density, compute dP = D - D_prev and max |dP| with the
//      reference's finiteness checks (one kernel, one status word);
//   2. skip an unchanged density unless a rebuild is forced;
//   3. build G from D (exact rebuild: first density, forced, or the
//      exact_rebuild_interval-th changed density) or dG from dP under the
//      delta density threshold (fused G density predicate);
//   4. next G = G_built or G + dG, with the non-finite checks;
//   5. commit by swapping buffers.
// Steps 1-4 write only scratch buffers, so any failure leaves the state as it
// was (the reference's strong guarantee).
#include <algorithm>
#include <memory>
#include <string>
#include <utility>

#include "jk_build.hpp"
#include "kernels.hpp"

using namespace tlno_gpu;

struct tlno_gpu_incremental {
    tlno_gpu_context* ctx = nullptr;
    tlno_gpu_incremental_options options{};
    std::unique_ptr<Plan2e> plan;
    int M = 0;
    long long n = 0;
    // committed state
    DeviceBuffer D, G;
    bool initialized = false;
    tlno_gpu_incremental_info info{};
    // scratch of one update
    DeviceBuffer D_in, delta, Gb, Gnext, J, K, D32, dmax, status;
    int fail_stage = 0;  // testing hook
};

namespace {

void check_options(const tlno_gpu_incremental_options& o) {
    if (o.exact_rebuild_interval == 0u)
        throw Error(TLNO_GPU_E_INVALID, "eri_ao_tensor_hgp: incremental exact_rebuild_interval must be >= 1.");
    const tlno_gpu_screening& b = o.base_options;
    if (!finite_bits(b.integral_threshold) || b.integral_threshold < 0.0)
        throw Error(TLNO_GPU_E_INVALID,
                    "eri_ao_tensor_hgp: incremental schwarz_threshold must be finite and >= 0.");
    if (!finite_bits(b.primitive_fastschwarz_threshold) || b.primitive_fastschwarz_threshold < 0.0)
        throw Error(TLNO_GPU_E_INVALID,
                    "eri_ao_tensor_hgp: incremental primitive_fastschwarz_threshold must be finite and >= 0.");
    if (!finite_bits(b.decay_threshold) || b.decay_threshold < 0.0)
        throw Error(TLNO_GPU_E_INVALID, "eri_ao_tensor_hgp: incremental decay_threshold must be finite and >= 0.");
    if (!finite_bits(b.density_threshold) || b.density_threshold < 0.0)
        throw Error(TLNO_GPU_E_INVALID,
                    "eri_ao_tensor_hgp: incremental base density_threshold must be finite and >= 0.");
    if (!finite_bits(b.mixed_threshold) || b.mixed_threshold < 0.0)
        throw Error(TLNO_GPU_E_INVALID, "tlno_gpu: mixed_threshold must be finite and >= 0.");
    if (b.integral_threshold != 0.0 && b.decay_threshold != 0.0)
        throw Error(TLNO_GPU_E_INVALID,
                    "eri_ao_tensor_hgp: incremental base options cannot combine Schwarz and decay screening.");
    if (!finite_bits(o.delta_density_threshold) || o.delta_density_threshold < 0.0)
        throw Error(TLNO_GPU_E_INVALID,
                    "eri_ao_tensor_hgp: incremental delta_density_threshold must be finite and >= 0.");
    if (!finite_bits(o.first_delta_density_threshold) || o.first_delta_density_threshold < 0.0)
        throw Error(TLNO_GPU_E_INVALID,
                    "eri_ao_tensor_hgp: incremental first_delta_density_threshold must be finite and >= 0.");
    if ((o.delta_density_threshold > 0.0 ||
         (o.use_first_delta_density_threshold && o.first_delta_density_threshold > 0.0)) &&
        b.decay_threshold > 0.0)
        throw Error(TLNO_GPU_E_INVALID,
                    "eri_ao_tensor_hgp: incremental delta-density screening cannot be combined with the heuristic "
                    "decay metric.");
}

unsigned int read_status(tlno_gpu_incremental* st, cudaStream_t s) {
    unsigned int v = 0;
    TLNO_CUDA(cudaMemcpyAsync(&v, st->status.ptr, sizeof(v), cudaMemcpyDeviceToHost, s));
    TLNO_CUDA(cudaStreamSynchronize(s));
    return v;
}

int update(tlno_gpu_incremental* st, const double* density, bool force, int flags) {
    if (!density) throw Error(TLNO_GPU_E_INVALID, "tlno_gpu: null argument");
    tlno_gpu_context* ctx = st->ctx;
    TLNO_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->stream;
    const long long n = st->n;
    const std::size_t bytes = sizeof(double) * static_cast<std::size_t>(std::max<long long>(n, 1));
    for (DeviceBuffer* b : {&st->D_in, &st->delta, &st->Gb, &st->Gnext, &st->J, &st->K}) b->alloc(bytes);
    st->dmax.alloc(16);
    st->status.alloc(16);
    // 1. stage D, dP and its checks
    if (flags & TLNO_GPU_DEVICE_PTRS)
        TLNO_CUDA(cudaMemcpyAsync(st->D_in.ptr, density, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    else
        TLNO_CUDA(cudaMemcpyAsync(st->D_in.ptr, density, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    launch_density_delta(st->D_in.as<double>(), st->initialized ? st->D.as<double>() : nullptr,
                         st->delta.as<double>(), n, st->status.as<unsigned int>(), st->dmax.as<double>(), s);
    double max_abs_delta = 0.0;
    TLNO_CUDA(cudaMemcpyAsync(&max_abs_delta, st->dmax.ptr, sizeof(double), cudaMemcpyDeviceToHost, s));
    const unsigned int dst = read_status(st, s);
    if (dst & 1u) throw Error(TLNO_GPU_E_INVALID, "eri_ao_tensor_hgp: incremental density contains a non-finite value.");
    if (dst & 2u) throw Error(TLNO_GPU_E_INVALID, "eri_ao_tensor_hgp: incremental density delta overflowed.");
    const bool unchanged = st->initialized && !(dst & 4u);
    // 2. an explicit force beats the unchanged fast path; an unchanged call
    // does not advance the cadence
    if (unchanged && !force) {
        st->info.updates++;
        st->info.skipped_updates++;
        st->info.last_status = TLNO_GPU_UPDATE_SKIPPED;
        st->info.last_max_abs_density_delta = 0.0;
        st->info.last_effective_density_threshold = 0.0;
        return TLNO_GPU_UPDATE_SKIPPED;
    }
    const bool periodic = st->initialized &&
                          st->info.updates_since_exact_rebuild >= st->options.exact_rebuild_interval - 1u;
    const bool exact = !st->initialized || force || periodic;
    tlno_gpu_screening bo = st->options.base_options;
    bo.density_threshold = 0.0;
    double eff = 0.0;
    if (!exact) {
        const bool first_after_exact = st->info.updates_since_exact_rebuild == 0u;
        eff = (st->options.use_first_delta_density_threshold && first_after_exact)
                  ? st->options.first_delta_density_threshold
                  : st->options.delta_density_threshold;
        bo.density_threshold = eff;
    }
    // 3. build G (or dG) from D (or dP); the builder validates its input
    const double* in = exact ? st->D_in.as<double>() : st->delta.as<double>();
    TLNO_CUDA(cudaMemsetAsync(st->status.ptr, 0, sizeof(unsigned int), s));
    launch_validate_density(in, st->M, st->status.as<unsigned int>(), s);
    const unsigned int vst = read_status(st, s);
    if (vst & 1u) throw Error(TLNO_GPU_E_INVALID, "eri_ao_tensor_hgp: density contains a non-finite value.");
    if (vst & 2u) throw Error(TLNO_GPU_E_INVALID, "eri_ao_tensor_hgp: density must be symmetric.");
    validate_build_combination(bo);
    if (st->fail_stage == 1) {
        st->fail_stage = 0;
        throw Error(TLNO_GPU_E_STATE, "tlno_gpu: injected incremental failure before the build");
    }
    if (bo.density_threshold > 0.0) ensure_density_tables(*st->plan);
    const bool mixed = flags & TLNO_GPU_MIXED;
    float* d32 = nullptr;
    if (mixed) {
        st->D32.alloc(sizeof(float) * static_cast<std::size_t>(std::max<long long>(n, 1)));
        d32 = st->D32.as<float>();
    }
    enqueue_jk(*st->plan, ctx->tune, spec_from(bo, true, true, mixed, true), in, st->J.as<double>(),
               st->K.as<double>(), n, st->M, st->dmax.as<double>(), d32, s);
    launch_combine_g(st->J.as<double>(), st->K.as<double>(), st->Gb.as<double>(), n, s);
    // 4. next G with the reference's non-finite checks
    launch_g_accumulate(exact ? nullptr : st->G.as<double>(), st->Gb.as<double>(), st->Gnext.as<double>(), n,
                        st->status.as<unsigned int>(), s);
    const unsigned int gst = read_status(st, s);
    if (exact && (gst & 3u))
        throw Error(TLNO_GPU_E_INVALID, "eri_ao_tensor_hgp: exact direct J/K rebuild produced a non-finite value.");
    if (gst & 1u)
        throw Error(TLNO_GPU_E_INVALID, "eri_ao_tensor_hgp: incremental dG build produced a non-finite value.");
    if (gst & 2u) throw Error(TLNO_GPU_E_INVALID, "eri_ao_tensor_hgp: incremental cached G overflowed.");
    if (st->fail_stage == 2) {
        st->fail_stage = 0;
        throw Error(TLNO_GPU_E_STATE, "tlno_gpu: injected incremental failure before the commit");
    }
    // 5. commit
    std::swap(st->D, st->D_in);
    std::swap(st->G, st->Gnext);
    st->initialized = true;
    st->info.initialized = 1;
    st->info.updates++;
    st->info.last_max_abs_density_delta = max_abs_delta;
    st->info.last_effective_density_threshold = eff;
    if (exact) {
        st->info.exact_rebuilds++;
        st->info.updates_since_exact_rebuild = 0;
        st->info.last_status = TLNO_GPU_UPDATE_EXACT;
    } else {
        st->info.incremental_updates++;
        st->info.updates_since_exact_rebuild++;
        st->info.last_status = TLNO_GPU_UPDATE_INCREMENTAL;
    }
    return st->info.last_status;
}

void copy_out(const tlno_gpu_incremental* st, const DeviceBuffer& src, double* dst, int flags) {
    if (!dst) throw Error(TLNO_GPU_E_INVALID, "tlno_gpu: null argument");
    if (!st->initialized) throw Error(TLNO_GPU_E_STATE, "tlno_gpu: incremental state holds no density yet");
    TLNO_CUDA(cudaSetDevice(st->ctx->device));
    const cudaMemcpyKind kind = (flags & TLNO_GPU_DEVICE_PTRS) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    TLNO_CUDA(cudaMemcpyAsync(dst, src.ptr, sizeof(double) * st->n, kind, st->ctx->stream));
    TLNO_CUDA(cudaStreamSynchronize(st->ctx->stream));
}

}  // namespace

extern "C" {

int tlno_gpu_incremental_create(tlno_gpu_context* ctx, const tlno_gpu_incremental_options* options,
                                tlno_gpu_incremental** out) {
    return run_guarded([&] {
        if (!ctx || !options || !out) throw Error(TLNO_GPU_E_INVALID, "tlno_gpu: null argument");
        *out = nullptr;
        check_options(*options);
        auto st = std::make_unique<tlno_gpu_incremental>();
        st->ctx = ctx;
        st->options = *options;
        // a full-density threshold would make an exact refresh depend on P
        st->options.base_options.density_threshold = 0.0;
        TLNO_CUDA(cudaSetDevice(ctx->device));
        st->plan = make_plan(ctx, st->options.base_options);
        st->M = ctx->basis.n_sph;
        st->n = static_cast<long long>(st->M) * st->M;
        *out = st.release();
    });
}

void tlno_gpu_incremental_destroy(tlno_gpu_incremental* st) {
    if (st && st->ctx) cudaSetDevice(st->ctx->device);
    delete st;
}

int tlno_gpu_incremental_update(tlno_gpu_incremental* st, const double* density, int force_exact_rebuild,
                                int flags) {
    int status = 0;
    const int rc = run_guarded([&] {
        if (!st) throw Error(TLNO_GPU_E_INVALID, "tlno_gpu: null argument");
        status = update(st, density, force_exact_rebuild != 0, flags);
    });
    return rc == TLNO_GPU_OK ? status : rc;
}

int tlno_gpu_incremental_g(const tlno_gpu_incremental* st, double* G, int flags) {
    return run_guarded([&] {
        if (!st) throw Error(TLNO_GPU_E_INVALID, "tlno_gpu: null argument");
        copy_out(st, st->G, G, flags);
    });
}

int tlno_gpu_incremental_density(const tlno_gpu_incremental* st, double* D, int flags) {
    return run_guarded([&] {
        if (!st) throw Error(TLNO_GPU_E_INVALID, "tlno_gpu: null argument");
        copy_out(st, st->D, D, flags);
    });
}

int tlno_gpu_incremental_info_get(const tlno_gpu_incremental* st, tlno_gpu_incremental_info* out) {
    return run_guarded([&] {
        if (!st || !out) throw Error(TLNO_GPU_E_INVALID, "tlno_gpu: null argument");
        *out = st->info;
    });
}

int tlno_gpu_incremental_reset(tlno_gpu_incremental* st) {
    return run_guarded([&] {
        if (!st) throw Error(TLNO_GPU_E_INVALID, "tlno_gpu: null argument");
        st->initialized = false;
        st->info = tlno_gpu_incremental_info{};
        st->fail_stage = 0;
    });
}

int tlno_gpu_incremental_fail_next_update(tlno_gpu_incremental* st, int stage) {
    return run_guarded([&] {
        if (!st || stage < 0 || stage > 2) throw Error(TLNO_GPU_E_INVALID, "tlno_gpu: invalid failure stage");
        st->fail_stage = stage;
    });
}

}  // extern "C"
