// extern "C" implementation of include/tlno_gpu.h.
//
// Every entry point catches all exceptions and turns them into a status
// code plus a thread-local message (the reference's exception texts are
// kept for the same conditions).  Buffers flagged TLNO_GPU_DEVICE_PTRS are
// used in place; host buffers are staged through context-owned device
// buffers on the context's stream.
#include "../../include/tlno_gpu.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <functional>
#include <memory>
#include <string>
#include <vector>

#include "engine.hpp"
#include "kernels.hpp"
#include "plan.hpp"
#include "tables.hpp"
#include "context.hpp"
#include "jk_build.hpp"

using namespace tlno_gpu;

namespace {

thread_local std::string g_error;

template <class F>
int guarded(F&& f) {
    try {
        f();
        return TLNO_GPU_OK;
    } catch (const Error& e) {
        g_error = e.what();
        return e.code;
    } catch (const std::bad_alloc&) {
        g_error = "tlno_gpu: host allocation failed";
        return TLNO_GPU_E_INVALID;
    } catch (const std::exception& e) {
        g_error = e.what();
        return TLNO_GPU_E_INVALID;
    } catch (...) {
        g_error = "tlno_gpu: unknown exception";
        return TLNO_GPU_E_INVALID;
    }
}

}  // namespace

int tlno_gpu::run_guarded(const std::function<void()>& f) { return guarded(f); }

namespace tlno_gpu {

void set_device(int device) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        throw Error(TLNO_GPU_E_CUDA, "tlno_gpu: no CUDA device available (there is no CPU fallback)");
    }
    if (device < 0 || device >= n) throw Error(TLNO_GPU_E_INVALID, "tlno_gpu: invalid device index");
    TLNO_CUDA(cudaSetDevice(device));
}

void validate_screening(const tlno_gpu_screening& o) {
    if (!finite_bits(o.integral_threshold) || o.integral_threshold < 0.0)
        throw Error(TLNO_GPU_E_INVALID, "eri_ao_tensor_hgp: schwarz_threshold must be finite and >= 0.");
    if (!finite_bits(o.decay_threshold) || o.decay_threshold < 0.0)
        throw Error(TLNO_GPU_E_INVALID, "eri_ao_tensor_hgp: decay_threshold must be finite and >= 0.");
    if (!finite_bits(o.primitive_fastschwarz_threshold) || o.primitive_fastschwarz_threshold < 0.0)
        throw Error(TLNO_GPU_E_INVALID,
                    "eri_ao_tensor_hgp: primitive_fastschwarz_threshold must be finite and >= 0.");
    if (!finite_bits(o.density_threshold) || o.density_threshold < 0.0)
        throw Error(TLNO_GPU_E_INVALID, "eri_ao_tensor_hgp: density_threshold must be finite and >= 0.");
    if (!finite_bits(o.mixed_threshold) || o.mixed_threshold < 0.0)
        throw Error(TLNO_GPU_E_INVALID, "tlno_gpu: mixed_threshold must be finite and >= 0.");
}

// Build-time combination rules of the reference's direct J/K route
// (direct_build.ipp:104-116, then rys_engine.ipp:18253-18262 for the
// specialised route whose single shell-level metric this engine follows).
void validate_build_combination(const tlno_gpu_screening& o) {
    if (o.density_threshold > 0.0 && o.decay_threshold > 0.0)
        throw Error(TLNO_GPU_E_INVALID,
                    "eri_ao_tensor_hgp: density screening requires Schwarz bounds and cannot be combined with "
                    "the heuristic decay metric.");
    if (o.integral_threshold != 0.0 && o.decay_threshold != 0.0)
        throw Error(TLNO_GPU_E_INVALID,
                    "eri_ao_tensor_hgp: pure-spherical Schwarz+decay screening is not part of the independent "
                    "decay checkpoint; select exactly one shell-level metric.");
}

// Host-side density contract (direct_build.ipp:25-96).
void validate_density_host(const double* D, int M) {
    constexpr double tol = 128.0 * 2.220446049250313e-16;
    for (int i = 0; i < M; ++i) {
        for (int j = 0; j <= i; ++j) {
            const double a = D[static_cast<std::size_t>(i) * M + j];
            if (!finite_bits(a)) throw Error(TLNO_GPU_E_INVALID, "eri_ao_tensor_hgp: density contains a non-finite value.");
            if (i == j) continue;
            const double b = D[static_cast<std::size_t>(j) * M + i];
            if (!finite_bits(b)) throw Error(TLNO_GPU_E_INVALID, "eri_ao_tensor_hgp: density contains a non-finite value.");
            const double sc = std::max({1.0, std::fabs(a), std::fabs(b)});
            if (std::fabs(a - b) > tol * sc) throw Error(TLNO_GPU_E_INVALID, "eri_ao_tensor_hgp: density must be symmetric.");
        }
    }
}



BuildSpec spec_from(const tlno_gpu_screening& o, bool want_j, bool want_k, bool mixed, bool fused_g) {
    BuildSpec b;
    b.want_j = want_j;
    b.want_k = want_k;
    b.mixed = mixed;
    b.mixed_threshold = o.mixed_threshold;
    b.den_thr = o.density_threshold;
    b.den_mode = o.density_threshold > 0.0 ? (fused_g ? 2 : 1) : 0;
    b.fs_thr2 = o.primitive_fastschwarz_threshold * o.primitive_fastschwarz_threshold;
    return b;
}

// Enqueues one J/K build on stream s over device buffers (the density tables
// of a density-screened build must be allocated before: ensure_density_tables).
void StreamFan::ensure(int n_aux) {
    TLNO_CUDA(cudaGetDevice(&device));
    while (static_cast<int>(aux.size()) < n_aux) {
        cudaStream_t st = nullptr;
        TLNO_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        aux.push_back(st);
    }
    while (static_cast<int>(ev.size()) < n_aux + 1) {
        cudaEvent_t e = nullptr;
        TLNO_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        ev.push_back(e);
    }
}

StreamFan::~StreamFan() {
    if (aux.empty() && ev.empty()) return;
    cudaSetDevice(device);
    for (cudaStream_t st : aux) cudaStreamDestroy(st);
    for (cudaEvent_t e : ev) cudaEventDestroy(e);
}

void enqueue_jk(Plan2e& plan, const Tuning& tune, const BuildSpec& spec, const double* dD, double* dJ,
                double* dK, long long total, int M_single, double* d_dmax, float* dD32, cudaStream_t s,
                StreamFan* fan) {
    const bool want_j = spec.want_j, want_k = spec.want_k, mixed = spec.mixed;
    TLNO_CUDA(cudaMemsetAsync(dJ, 0, sizeof(double) * total, s));
    TLNO_CUDA(cudaMemsetAsync(dK, 0, sizeof(double) * total, s));
    TLNO_CUDA(cudaMemsetAsync(plan.d_counters.ptr, 0, sizeof(int) * 2 * plan.combos.size(), s));
    if (mixed) launch_absmax_f32(dD, total, d_dmax, dD32, s);
    dev::DensityScreen den{};
    if (spec.den_mode) {
        if (!plan.d_rho_blk.ptr || !plan.d_rho_max.ptr)
            throw Error(TLNO_GPU_E_STATE, "tlno_gpu: density-screen tables not allocated");
        const bool multi = plan.n_mol > 1;
        launch_density_blocks(dD, multi ? plan.d_mol_mat_off.as<long long>() : nullptr,
                              multi ? plan.d_mol_M.as<int>() : nullptr, M_single, plan.d_shell_sph.as<int>(),
                              plan.d_shell_L.as<int>(), multi ? plan.d_mol_shell_off.as<int>() : nullptr,
                              multi ? plan.d_mol_ns.as<int>() : nullptr, plan.mol_ns.empty() ? 0 : plan.mol_ns[0],
                              plan.n_mol, plan.max_ns2, multi ? plan.d_rho_off.as<long long>() : nullptr,
                              plan.d_rho_blk.as<double>(), plan.d_rho_max.as<double>(), s);
        den.mode = spec.den_mode;
        den.thr = spec.den_thr;
        den.rho_blk = plan.d_rho_blk.as<double>();
        den.rho_off = multi ? plan.d_rho_off.as<long long>() : nullptr;
        den.rho_max = plan.d_rho_max.as<double>();
    }
    const dev::PlanView pv = plan.view();
    int sms = 0, devid = 0;
    TLNO_CUDA(cudaGetDevice(&devid));
    TLNO_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, devid));
    // Class launches over `nst` streams: fork after the shared prologue
    // (zeroing, max|D|, density tables), each class on the stream with the
    // least flops so far (largest classes first), join before the
    // symmetrisation.  J and K take FP64 atomics, so the order is free.
    const int nst = (fan && tune.streams > 1) ? std::min(tune.streams, 4) : 1;
    std::vector<cudaStream_t> st(1, s);
    std::vector<int> stream_of(plan.combos.size(), 0);
    if (nst > 1) {
        fan->ensure(nst - 1);
        TLNO_CUDA(cudaEventRecord(fan->ev[0], s));
        for (int k = 0; k < nst - 1; ++k) {
            TLNO_CUDA(cudaStreamWaitEvent(fan->aux[k], fan->ev[0], 0));
            st.push_back(fan->aux[k]);
        }
        std::vector<std::size_t> order(plan.combos.size());
        for (std::size_t i = 0; i < order.size(); ++i) order[i] = i;
        std::stable_sort(order.begin(), order.end(),
                         [&](std::size_t a, std::size_t b) { return plan.combos[a].flops > plan.combos[b].flops; });
        std::vector<double> load(nst, 0.0);
        for (std::size_t i : order) {
            const int k = static_cast<int>(std::min_element(load.begin(), load.end()) - load.begin());
            stream_of[i] = k;
            load[k] += plan.combos[i].flops;
        }
    }
    for (std::size_t ci = 0; ci < plan.combos.size(); ++ci) {
        ComboSchedule& cs = plan.combos[ci];
        cudaStream_t cs_stream = st[stream_of[ci]];
        dev::ClassLaunch cl{};
        cl.la = cs.la; cl.lb = cs.lb; cl.lc = cs.lc; cl.ld = cs.ld;
        cl.same = (cs.X == cs.Y);
        cl.bb = cs.bb;
        cl.bk = cs.bk;
        cl.blocks = cs.d_blocks.as<dev::BlockDesc>();
        cl.bra_list = cs.d_bra_list.as<int>();
        cl.tile_prefix = cs.d_prefix.as<int>();
        cl.n_blocks = static_cast<int>(cs.blocks.size());
        cl.tile_begin = 0;
        cl.tile_end = cs.n_tiles;
        cl.tau = plan.tau;
        cl.tau_mix = spec.mixed_threshold * cs.mix_scale;
        cl.chunk = cs.chunk;
        cl.den = den;
        cl.fs_thr2 = spec.fs_thr2;
        cl.M_shells = plan.mol_ns.empty() ? 0 : plan.mol_ns[0];
        cl.dmax = d_dmax;
        cl.dens = dD;
        cl.dens32 = dD32;
        cl.J = dJ;
        cl.K = dK;
        cl.M = M_single;
        cl.want_j = want_j;
        cl.want_k = want_k;
        const int grid = sms * tune.grid_mult;
        // a class whose split multiplier is 0 stays FP64 in a mixed build
        // (one launch, no FP32 pass)
        const bool split = mixed && cs.mix_scale > 0.0;
        const int passes = split ? 2 : 1;
        for (int pass = 0; pass < passes; ++pass) {
            cl.prec_mode = split ? (pass + 1) : 0;
            cl.counter = plan.d_counters.as<int>() + 2 * ci + pass;
            const bool fp32 = split && pass == 1;
            if (cs.fast) {
                launch_eri_jk_fast(pv, cl, fp32, grid, cs_stream);
            } else {
                launch_eri_jk_generic(pv, cl, fp32, tune.generic_warps, grid, cs_stream);
            }
        }
    }
    if (nst > 1) {
        for (int k = 0; k < nst - 1; ++k) {
            TLNO_CUDA(cudaEventRecord(fan->ev[k + 1], fan->aux[k]));
            TLNO_CUDA(cudaStreamWaitEvent(s, fan->ev[k + 1], 0));
        }
    }
    if (plan.n_mol > 1) {
        int maxm = 0;
        for (int m : plan.mol_M) maxm = std::max(maxm, m);
        if (want_j) launch_symmetrize(dJ, plan.d_mol_mat_off.as<long long>(), plan.d_mol_M.as<int>(), plan.n_mol, maxm, s);
        if (want_k) launch_symmetrize(dK, plan.d_mol_mat_off.as<long long>(), plan.d_mol_M.as<int>(), plan.n_mol, maxm, s);
    } else {
        if (want_j) launch_symmetrize_single(dJ, M_single, s);
        if (want_k) launch_symmetrize_single(dK, M_single, s);
    }
}

}  // namespace tlno_gpu

void tlno_gpu::set_last_error(const std::string& message) { g_error = message; }

namespace {

void init_context(tlno_gpu_context* c) {
    set_device(c->device);
    ensure_device_tables();
    noalloc_prepare(c->device);
    TLNO_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    const Basis& b = c->basis;
    const int ns = static_cast<int>(b.shells.size());
    std::vector<double> xyz(3 * std::max(ns, 1));
    std::vector<int> L(std::max(ns, 1)), np(std::max(ns, 1)), po(std::max(ns, 1)), sph(std::max(ns, 1));
    for (int i = 0; i < ns; ++i) {
        for (int k = 0; k < 3; ++k) xyz[3 * i + k] = b.shells[i].center[k];
        L[i] = b.shells[i].L;
        np[i] = b.shells[i].nprim;
        po[i] = b.shells[i].prim_offset;
        sph[i] = b.shells[i].sph_offset;
    }
    auto up = [&](DeviceBuffer& d, const void* src, std::size_t bytes) {
        d.alloc(std::max<std::size_t>(bytes, 16));
        if (bytes) TLNO_CUDA(cudaMemcpy(d.ptr, src, bytes, cudaMemcpyHostToDevice));
    };
    up(c->d_shell_xyz, xyz.data(), xyz.size() * sizeof(double));
    up(c->d_shell_L, L.data(), L.size() * sizeof(int));
    up(c->d_shell_nprim, np.data(), np.size() * sizeof(int));
    up(c->d_shell_prim, po.data(), po.size() * sizeof(int));
    up(c->d_shell_sph, sph.data(), sph.size() * sizeof(int));
    up(c->d_exps, b.exps.data(), b.exps.size() * sizeof(double));
    up(c->d_crad, b.c_radial.data(), b.c_radial.size() * sizeof(double));
    up(c->d_comp_coef, b.comp_coef.data(), b.comp_coef.size() * sizeof(double));
    up(c->d_comp_off, b.comp_offset.data(), b.comp_offset.size() * sizeof(int));
}

// (Re)builds the context's two-electron plan for the shell-level screen of
// `o` (Schwarz threshold or decay metric).
void replan(tlno_gpu_context* ctx, const tlno_gpu_screening& o) {
    TLNO_CUDA(cudaSetDevice(ctx->device));
    if (ctx->graph_exec) { cudaGraphExecDestroy(ctx->graph_exec); ctx->graph_exec = nullptr; }
    if (ctx->graph) { cudaGraphDestroy(ctx->graph); ctx->graph = nullptr; }
    ctx->plan = make_plan(ctx, o);
    ctx->screening = o;
}

}  // namespace

namespace tlno_gpu {

std::unique_ptr<Plan2e> make_plan(const tlno_gpu_context* ctx, const tlno_gpu_screening& o) {
    if (ctx->basis.n_sph > 65535)
        throw Error(TLNO_GPU_E_INVALID, "eri_ao_tensor_hgp: direct J/K pair tables assume M <= 65535.");
    auto plan = std::make_unique<Plan2e>();
    std::vector<MolPairs> mp;
    const double tau = o.decay_threshold > 0.0 ? o.decay_threshold : o.integral_threshold;
    mp.push_back(build_mol_pairs(ctx->basis, o.integral_threshold, ctx->stream, o.decay_threshold));
    build_plan(*plan, {&ctx->basis}, std::move(mp), tau, ctx->tune, ctx->stream);
    plan->decay_metric = o.decay_threshold > 0.0;
    return plan;
}

void ensure_work(JkWork& w, long long total) {
    const std::size_t bytes = sizeof(double) * std::max<long long>(total, 1);
    w.D.alloc(bytes);
    w.J.alloc(bytes);
    w.K.alloc(bytes);
    w.dmax.alloc(16);
    w.status.alloc(16);
}

}  // namespace tlno_gpu

namespace {

// One J/K build of a context with screening options `o` (the reference's
// build-time ScreeningOptions): a shell-level screen other than the plan's
// re-plans; density and primitive FASTSCHWARZ screening apply to this build.
void run_jk(tlno_gpu_context* ctx, const double* density, double* J, double* K, double* G, int flags,
            const tlno_gpu_screening& o) {
    if (!ctx || !density) throw Error(TLNO_GPU_E_INVALID, "tlno_gpu: null argument");
    if (!ctx->plan) throw Error(TLNO_GPU_E_STATE, "tlno_gpu: no plan; call tlno_gpu_plan first");
    const bool want_g = flags & TLNO_GPU_WANT_G;
    const bool out_j = flags & TLNO_GPU_WANT_J, out_k = flags & TLNO_GPU_WANT_K;
    if (!out_j && !out_k && !want_g) throw Error(TLNO_GPU_E_INVALID, "tlno_gpu: no output selected");
    if (out_j && !J) throw Error(TLNO_GPU_E_INVALID, "tlno_gpu: null J");
    if (out_k && !K) throw Error(TLNO_GPU_E_INVALID, "tlno_gpu: null K");
    if (want_g && !G) throw Error(TLNO_GPU_E_INVALID, "tlno_gpu: null G");
    const bool dev_ptrs = flags & TLNO_GPU_DEVICE_PTRS;
    const bool mixed = flags & TLNO_GPU_MIXED;
    const int M = ctx->basis.n_sph;
    const long long n = static_cast<long long>(M) * M;
    TLNO_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->stream;
    // density contract first, as the reference validates P before any option
    // combination (direct_build.ipp:67-81)
    const double* dD = density;
    ensure_work(ctx->w, n);
    if (!dev_ptrs) {
        if (!(flags & TLNO_GPU_NO_VALIDATE)) validate_density_host(density, M);
        TLNO_CUDA(cudaMemcpyAsync(ctx->w.D.ptr, density, sizeof(double) * n, cudaMemcpyHostToDevice, s));
        dD = ctx->w.D.as<double>();
    } else if (!(flags & TLNO_GPU_NO_VALIDATE)) {
        TLNO_CUDA(cudaMemsetAsync(ctx->w.status.ptr, 0, sizeof(unsigned int), s));
        launch_validate_density(dD, M, ctx->w.status.as<unsigned int>(), s);
        unsigned int st = 0;
        TLNO_CUDA(cudaMemcpyAsync(&st, ctx->w.status.ptr, sizeof(st), cudaMemcpyDeviceToHost, s));
        TLNO_CUDA(cudaStreamSynchronize(s));
        if (st & 1u) throw Error(TLNO_GPU_E_INVALID, "eri_ao_tensor_hgp: density contains a non-finite value.");
        if (st & 2u) throw Error(TLNO_GPU_E_INVALID, "eri_ao_tensor_hgp: density must be symmetric.");
    }
    validate_build_combination(o);
    if (o.integral_threshold != ctx->screening.integral_threshold ||
        o.decay_threshold != ctx->screening.decay_threshold) {
        const double keep_mixed = ctx->screening.mixed_threshold;
        replan(ctx, o);
        ctx->screening.mixed_threshold = keep_mixed;
    }
    const bool den = o.density_threshold > 0.0;
    if (den) ensure_density_tables(*ctx->plan);
    float* d32 = nullptr;
    if (mixed) {
        ctx->w.D32.alloc(sizeof(float) * n);
        d32 = ctx->w.D32.as<float>();
    }
    tlno_gpu_screening eo = o;
    eo.mixed_threshold = ctx->screening.mixed_threshold;
    // Without density screening one pass serves J, K and G.  With it, J and K
    // keep their own predicates (build_coulomb_j / build_exchange_k) and G the
    // fused one (build_rhf_g), so G takes its own pass when J or K is also
    // requested.
    const bool pass_jk = out_j || out_k || !den;
    double* dJ = (dev_ptrs && out_j) ? J : ctx->w.J.as<double>();
    double* dK = (dev_ptrs && out_k) ? K : ctx->w.K.as<double>();
    if (pass_jk) {
        const bool pj = den ? out_j : (out_j || want_g);
        const bool pk = den ? out_k : (out_k || want_g);
        enqueue_jk(*ctx->plan, ctx->tune, spec_from(eo, pj, pk, mixed, false), dD, dJ, dK, n, M,
                   ctx->w.dmax.as<double>(), d32, s, &ctx->fan);
        if (!dev_ptrs) {
            if (out_j) TLNO_CUDA(cudaMemcpyAsync(J, dJ, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
            if (out_k) TLNO_CUDA(cudaMemcpyAsync(K, dK, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
        }
    }
    if (want_g) {
        double* gJ = dJ;
        double* gK = dK;
        if (den) {
            gJ = ctx->w.J.as<double>();
            gK = ctx->w.K.as<double>();
            enqueue_jk(*ctx->plan, ctx->tune, spec_from(eo, true, true, mixed, true), dD, gJ, gK, n, M,
                       ctx->w.dmax.as<double>(), d32, s, &ctx->fan);
        }
        double* dG = G;
        if (!dev_ptrs) {
            ctx->w.G.alloc(sizeof(double) * std::max<long long>(n, 1));
            dG = ctx->w.G.as<double>();
        }
        launch_combine_g(gJ, gK, dG, n, s);
        if (!dev_ptrs) TLNO_CUDA(cudaMemcpyAsync(G, dG, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
    }
    TLNO_CUDA(cudaStreamSynchronize(s));
}

}  // namespace

extern "C" {

const char* tlno_gpu_last_error(void) { return g_error.c_str(); }

int tlno_gpu_version(void) { return 10000; }

int tlno_gpu_device_count(int* count) {
    return guarded([&] {
        int n = 0;
        if (cudaGetDeviceCount(&n) != cudaSuccess) {
            cudaGetLastError();
            n = 0;
        }
        *count = n;
    });
}

int tlno_gpu_create(int n_shells, const double* centers, const int* L, const int* nprim,
                    const double* exps, const double* coefs, int natom, const int* Z,
                    const double* atom_xyz, int device, tlno_gpu_context** out) {
    return guarded([&] {
        if (!out) throw Error(TLNO_GPU_E_INVALID, "tlno_gpu: null output handle");
        *out = nullptr;
        auto c = std::make_unique<tlno_gpu_context>();
        c->device = device;
        c->basis = basis_from_raw(n_shells, centers, L, nprim, exps, coefs, natom, Z, atom_xyz);
        init_context(c.get());
        *out = c.release();
    });
}

int tlno_gpu_create_from_components(int n_components, const double* centers, const int* ang,
                                    const int* nprim, const double* exps, const double* coefs,
                                    int natom, const int* Z, const double* atom_xyz, int device,
                                    tlno_gpu_context** out) {
    return guarded([&] {
        if (!out) throw Error(TLNO_GPU_E_INVALID, "tlno_gpu: null output handle");
        *out = nullptr;
        auto c = std::make_unique<tlno_gpu_context>();
        c->device = device;
        c->basis = basis_from_components(n_components, centers, ang, nprim, exps, coefs, natom, Z, atom_xyz);
        init_context(c.get());
        *out = c.release();
    });
}

void tlno_gpu_destroy(tlno_gpu_context* ctx) { delete ctx; }

int tlno_gpu_n_sph(const tlno_gpu_context* ctx) { return ctx ? ctx->basis.n_sph : -1; }
int tlno_gpu_n_shells(const tlno_gpu_context* ctx) {
    return ctx ? static_cast<int>(ctx->basis.shells.size()) : -1;
}

int tlno_gpu_plan(tlno_gpu_context* ctx, const tlno_gpu_screening* options) {
    return guarded([&] {
        if (!ctx) throw Error(TLNO_GPU_E_INVALID, "tlno_gpu: null context");
        tlno_gpu_screening o = options ? *options : tlno_gpu_screening{1e-12, 0, 0, 0, 1e-9};
        validate_screening(o);
        replan(ctx, o);
    });
}

int tlno_gpu_plan_profile(const tlno_gpu_context* ctx, tlno_gpu_profile* out) {
    return guarded([&] {
        if (!ctx || !out) throw Error(TLNO_GPU_E_INVALID, "tlno_gpu: null argument");
        if (!ctx->plan) throw Error(TLNO_GPU_E_STATE, "tlno_gpu: no plan; call tlno_gpu_plan first");
        const Plan2e& p = *ctx->plan;
        out->M = ctx->basis.n_sph;
        out->n_shells = static_cast<int>(ctx->basis.shells.size());
        out->shell_pairs = p.total_pairs;
        out->kept_pairs = p.kept_pairs;
        out->quartets = p.total_quartets;
        out->primitive_quartets = p.total_prim_quartets;
        out->flops = p.total_flops;
        out->n_class_launches = static_cast<int>(p.combos.size());
    });
}

int tlno_gpu_jk(tlno_gpu_context* ctx, const double* density, double* J, double* K, double* G, int flags) {
    return guarded([&] {
        if (!ctx) throw Error(TLNO_GPU_E_INVALID, "tlno_gpu: null argument");
        run_jk(ctx, density, J, K, G, flags, ctx->screening);
    });
}

int tlno_gpu_jk_with_options(tlno_gpu_context* ctx, const double* density, double* J, double* K, double* G,
                             int flags, const tlno_gpu_screening* options) {
    return guarded([&] {
        if (!ctx || !options) throw Error(TLNO_GPU_E_INVALID, "tlno_gpu: null argument");
        validate_screening(*options);
        run_jk(ctx, density, J, K, G, flags, *options);
    });
}

int tlno_gpu_eri_checksum(tlno_gpu_context* ctx, double* checksum, double* ms) {
    return guarded([&] {
        if (!ctx || !checksum) throw Error(TLNO_GPU_E_INVALID, "tlno_gpu: null argument");
        if (!ctx->plan) throw Error(TLNO_GPU_E_STATE, "tlno_gpu: no plan; call tlno_gpu_plan first");
        TLNO_CUDA(cudaSetDevice(ctx->device));
        cudaStream_t s = ctx->stream;
        Plan2e& plan = *ctx->plan;
        ensure_work(ctx->w, 1);
        double* d_sum = ctx->w.dmax.as<double>();
        int sms = 0;
        TLNO_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
        const dev::PlanView pv = plan.view();
        cudaEvent_t e0, e1;
        TLNO_CUDA(cudaEventCreate(&e0));
        TLNO_CUDA(cudaEventCreate(&e1));
        TLNO_CUDA(cudaMemsetAsync(d_sum, 0, sizeof(double), s));
        TLNO_CUDA(cudaMemsetAsync(plan.d_counters.ptr, 0, sizeof(int) * 2 * plan.combos.size(), s));
        TLNO_CUDA(cudaEventRecord(e0, s));
        for (std::size_t ci = 0; ci < plan.combos.size(); ++ci) {
            ComboSchedule& cs = plan.combos[ci];
            dev::ClassLaunch cl{};
            cl.la = cs.la; cl.lb = cs.lb; cl.lc = cs.lc; cl.ld = cs.ld;
            cl.same = (cs.X == cs.Y);
            cl.bb = cs.bb;
            cl.bk = cs.bk;
            cl.blocks = cs.d_blocks.as<dev::BlockDesc>();
            cl.bra_list = cs.d_bra_list.as<int>();
            cl.tile_prefix = cs.d_prefix.as<int>();
            cl.n_blocks = static_cast<int>(cs.blocks.size());
            cl.tile_begin = 0;
            cl.tile_end = cs.n_tiles;
            cl.tau = plan.tau;
            cl.dmax = d_sum;
            cl.M = ctx->basis.n_sph;
            cl.want_j = 0;
            cl.want_k = 0;
            cl.checksum = d_sum;
            cl.counter = plan.d_counters.as<int>() + 2 * ci;
            const int grid = sms * ctx->tune.grid_mult;
            if (cs.fast)
                launch_eri_jk_fast(pv, cl, false, grid, s);
            else
                launch_eri_jk_generic(pv, cl, false, ctx->tune.generic_warps, grid, s);
        }
        TLNO_CUDA(cudaEventRecord(e1, s));
        TLNO_CUDA(cudaMemcpyAsync(checksum, d_sum, sizeof(double), cudaMemcpyDeviceToHost, s));
        TLNO_CUDA(cudaStreamSynchronize(s));
        float t = 0.f;
        TLNO_CUDA(cudaEventElapsedTime(&t, e0, e1));
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (ms) *ms = t;
    });
}

int tlno_gpu_set_onee_thresholds(tlno_gpu_context* ctx, double group_pair_decay_eps, double nuclear_screen_eps) {
    return guarded([&] {
        if (!ctx) throw Error(TLNO_GPU_E_INVALID, "tlno_gpu: null context");
        if (!finite_bits(group_pair_decay_eps) || group_pair_decay_eps < 0 || !finite_bits(nuclear_screen_eps) ||
            nuclear_screen_eps < 0)
            throw Error(TLNO_GPU_E_INVALID, "tlno_gpu: screening thresholds must be finite and >= 0");
        ctx->onee_decay_eps = group_pair_decay_eps;
        ctx->onee_nuclear_eps = nuclear_screen_eps;
        ctx->onee_state = -1;
    });
}

int tlno_gpu_set_mixed_threshold(tlno_gpu_context* ctx, double mixed_threshold) {
    return guarded([&] {
        if (!ctx) throw Error(TLNO_GPU_E_INVALID, "tlno_gpu: null context");
        if (!finite_bits(mixed_threshold) || mixed_threshold < 0.0)
            throw Error(TLNO_GPU_E_INVALID, "tlno_gpu: mixed_threshold must be finite and >= 0.");
        ctx->screening.mixed_threshold = mixed_threshold;
    });
}

int tlno_gpu_onee(tlno_gpu_context* ctx, double* S, double* T, double* V, int screening, int flags) {
    return guarded([&] {
        if (!ctx || !S || !T || !V) throw Error(TLNO_GPU_E_INVALID, "tlno_gpu: null argument");
        TLNO_CUDA(cudaSetDevice(ctx->device));
        cudaStream_t s = ctx->stream;
        const int M = ctx->basis.n_sph;
        const long long n = static_cast<long long>(M) * M;
        const int state = screening ? 1 : 0;
        if (ctx->onee_state != state) {
            build_onee_plan(ctx->onee, ctx->basis, screening ? ctx->onee_decay_eps : 0.0,
                            screening ? ctx->onee_nuclear_eps : 0.0);
            auto up = [&](DeviceBuffer& d, const void* src, std::size_t bytes) {
                d.alloc(std::max<std::size_t>(bytes, 16));
                if (bytes) TLNO_CUDA(cudaMemcpyAsync(d.ptr, src, bytes, cudaMemcpyHostToDevice, s));
            };
            up(ctx->onee.d_pairs, ctx->onee.pairs.data(), ctx->onee.pairs.size() * sizeof(dev::OneePair));
            up(ctx->onee.d_maxc, ctx->onee.maxc.data(), ctx->onee.maxc.size() * sizeof(double));
            up(ctx->onee.d_nuc, ctx->onee.nuc.data(), ctx->onee.nuc.size() * sizeof(double));
            ctx->onee_state = state;
        }
        const bool dev_ptrs = flags & TLNO_GPU_DEVICE_PTRS;
        double *dS = S, *dT = T, *dV = V;
        if (!dev_ptrs) {
            ctx->d_S.alloc(sizeof(double) * std::max<long long>(n, 1));
            ctx->d_T.alloc(sizeof(double) * std::max<long long>(n, 1));
            ctx->d_V.alloc(sizeof(double) * std::max<long long>(n, 1));
            dS = ctx->d_S.as<double>();
            dT = ctx->d_T.as<double>();
            dV = ctx->d_V.as<double>();
        }
        TLNO_CUDA(cudaMemsetAsync(dS, 0, sizeof(double) * n, s));
        TLNO_CUDA(cudaMemsetAsync(dT, 0, sizeof(double) * n, s));
        TLNO_CUDA(cudaMemsetAsync(dV, 0, sizeof(double) * n, s));
        dev::OneeLaunch L{};
        L.shell_xyz = ctx->d_shell_xyz.as<double>();
        L.shell_L = ctx->d_shell_L.as<int>();
        L.shell_nprim = ctx->d_shell_nprim.as<int>();
        L.shell_prim = ctx->d_shell_prim.as<int>();
        L.shell_sph = ctx->d_shell_sph.as<int>();
        L.exps = ctx->d_exps.as<double>();
        L.c_radial = ctx->d_crad.as<double>();
        L.maxc = ctx->onee.d_maxc.as<double>();
        L.comp_coef = ctx->d_comp_coef.as<double>();
        L.comp_off = ctx->d_comp_off.as<int>();
        L.pairs = ctx->onee.d_pairs.as<dev::OneePair>();
        L.n_pairs = static_cast<int>(ctx->onee.pairs.size());
        L.nuc = ctx->onee.d_nuc.as<double>();
        L.n_nuc = static_cast<int>(ctx->onee.nuc.size() / 4);
        L.screen_thr = ctx->onee.screen_thr;
        L.M = M;
        L.S = dS;
        L.T = dT;
        L.V = dV;
        launch_onee(L, s);
        if (!dev_ptrs) {
            TLNO_CUDA(cudaMemcpyAsync(S, dS, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
            TLNO_CUDA(cudaMemcpyAsync(T, dT, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
            TLNO_CUDA(cudaMemcpyAsync(V, dV, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
        }
        TLNO_CUDA(cudaStreamSynchronize(s));
    });
}

int tlno_gpu_eri_blocks(tlno_gpu_context* ctx, int n_quartets, const int* shells4, const long long* offsets,
                        double* out) {
    return guarded([&] {
        if (!ctx || (n_quartets > 0 && (!shells4 || !offsets || !out)))
            throw Error(TLNO_GPU_E_INVALID, "tlno_gpu: null argument");
        TLNO_CUDA(cudaSetDevice(ctx->device));
        cudaStream_t s = ctx->stream;
        const Basis& b = ctx->basis;
        const int ns = static_cast<int>(b.shells.size());
        // Ad-hoc pair table: bra (A,B) and ket (C,D) of every quartet in the
        // requested orientation.
        std::vector<int> pA, pB, pnp, poff;
        std::vector<dev::DPrimPair> prim;
        long long total_out = 0;
        std::vector<std::vector<int>> by_class(625);
        for (int q = 0; q < n_quartets; ++q) {
            const int* sh = shells4 + 4 * q;
            for (int k = 0; k < 4; ++k)
                if (sh[k] < 0 || sh[k] >= ns) throw Error(TLNO_GPU_E_INVALID, "tlno_gpu: shell index out of range");
            const int la = b.shells[sh[0]].L, lb = b.shells[sh[1]].L, lc = b.shells[sh[2]].L, ld = b.shells[sh[3]].L;
            for (int side = 0; side < 2; ++side) {
                const int X = sh[2 * side], Y = sh[2 * side + 1];
                pA.push_back(X);
                pB.push_back(Y);
                poff.push_back(static_cast<int>(prim.size()));
                const std::size_t before = prim.size();
                primitive_pairs(b, X, Y, prim);
                pnp.push_back(static_cast<int>(prim.size() - before));
            }
            by_class[((la * 5 + lb) * 5 + lc) * 5 + ld].push_back(q);
            total_out = std::max<long long>(total_out, offsets[q] + static_cast<long long>(n_sph(la)) * n_sph(lb) *
                                                                     n_sph(lc) * n_sph(ld));
        }
        if (n_quartets == 0) return;
        std::vector<double> xyz(3 * ns);
        std::vector<int> Ls(ns), sph(ns);
        for (int i = 0; i < ns; ++i) {
            for (int k = 0; k < 3; ++k) xyz[3 * i + k] = b.shells[i].center[k];
            Ls[i] = b.shells[i].L;
            sph[i] = b.shells[i].sph_offset;
        }
        DeviceBuffer d_xyz, d_L, d_sph, d_A, d_B, d_np, d_off, d_prim, d_qb, d_qk, d_oo, d_out;
        auto up = [&](DeviceBuffer& d, const void* src, std::size_t bytes) {
            d.alloc(std::max<std::size_t>(bytes, 16));
            if (bytes) TLNO_CUDA(cudaMemcpyAsync(d.ptr, src, bytes, cudaMemcpyHostToDevice, s));
        };
        up(d_xyz, xyz.data(), xyz.size() * sizeof(double));
        up(d_L, Ls.data(), Ls.size() * sizeof(int));
        up(d_sph, sph.data(), sph.size() * sizeof(int));
        up(d_A, pA.data(), pA.size() * sizeof(int));
        up(d_B, pB.data(), pB.size() * sizeof(int));
        up(d_np, pnp.data(), pnp.size() * sizeof(int));
        up(d_off, poff.data(), poff.size() * sizeof(int));
        up(d_prim, prim.data(), prim.size() * sizeof(dev::DPrimPair));
        d_out.alloc(sizeof(double) * std::max<long long>(total_out, 1));
        dev::PlanView pv{};
        pv.shell_xyz = d_xyz.as<double>();
        pv.shell_L = d_L.as<int>();
        pv.shell_sph = d_sph.as<int>();
        pv.pair_A = d_A.as<int>();
        pv.pair_B = d_B.as<int>();
        pv.pair_nprim = d_np.as<int>();
        pv.pair_prim_off = d_off.as<int>();
        pv.prim = d_prim.as<dev::DPrimPair>();
        std::vector<int> qb, qk;
        std::vector<long long> oo;
        std::vector<int> cls_begin;
        std::vector<int> cls_key;
        for (int key = 0; key < 625; ++key) {
            if (by_class[key].empty()) continue;
            cls_begin.push_back(static_cast<int>(qb.size()));
            cls_key.push_back(key);
            for (int q : by_class[key]) {
                qb.push_back(2 * q);
                qk.push_back(2 * q + 1);
                oo.push_back(offsets[q]);
            }
        }
        cls_begin.push_back(static_cast<int>(qb.size()));
        up(d_qb, qb.data(), qb.size() * sizeof(int));
        up(d_qk, qk.data(), qk.size() * sizeof(int));
        up(d_oo, oo.data(), oo.size() * sizeof(long long));
        for (std::size_t c = 0; c + 1 < cls_begin.size(); ++c) {
            const int key = cls_key[c];
            dev::ClassLaunch cl{};
            cl.la = key / 125;
            cl.lb = (key / 25) % 5;
            cl.lc = (key / 5) % 5;
            cl.ld = key % 5;
            cl.q_bra = d_qb.as<int>() + cls_begin[c];
            cl.q_ket = d_qk.as<int>() + cls_begin[c];
            cl.out_off = d_oo.as<long long>() + cls_begin[c];
            cl.n_quartets = cls_begin[c + 1] - cls_begin[c];
            cl.out = d_out.as<double>();
            launch_eri_store(pv, cl, s);
        }
        TLNO_CUDA(cudaMemcpyAsync(out, d_out.ptr, sizeof(double) * total_out, cudaMemcpyDeviceToHost, s));
        TLNO_CUDA(cudaStreamSynchronize(s));
    });
}

int tlno_gpu_schwarz(const tlno_gpu_context* ctx, double* out) {
    return guarded([&] {
        if (!ctx || !out) throw Error(TLNO_GPU_E_INVALID, "tlno_gpu: null argument");
        if (!ctx->plan) throw Error(TLNO_GPU_E_STATE, "tlno_gpu: no plan; call tlno_gpu_plan first");
        const auto& q = ctx->plan->mol_pairs[0].Q_canonical;
        std::copy(q.begin(), q.end(), out);
    });
}

int tlno_gpu_boys(int device, int n, int maxn, const double* x, double* out) {
    return guarded([&] {
        if (n < 0 || maxn < 0 || maxn > 33) throw Error(TLNO_GPU_E_INVALID, "tlno_gpu: boys order must be 0..33");
        for (int i = 0; i < n; ++i)
            if (!finite_bits(x[i]) || x[i] < 0.0) throw Error(TLNO_GPU_E_INVALID, "tlno_gpu: boys argument must be finite and >= 0");
        set_device(device);
        ensure_device_tables();
        if (n == 0) return;
        DeviceBuffer dx, dout;
        dx.alloc(sizeof(double) * n);
        dout.alloc(sizeof(double) * n * (maxn + 1));
        TLNO_CUDA(cudaMemcpy(dx.ptr, x, sizeof(double) * n, cudaMemcpyHostToDevice));
        launch_boys_test(dx.as<double>(), n, maxn, dout.as<double>(), 0);
        TLNO_CUDA(cudaMemcpy(out, dout.ptr, sizeof(double) * n * (maxn + 1), cudaMemcpyDeviceToHost));
    });
}

int tlno_gpu_rys(int device, int n, int nroots, const double* T, double* roots, double* weights, int fp32) {
    return guarded([&] {
        if (n < 0 || nroots < 1 || nroots > kRysMaxN) throw Error(TLNO_GPU_E_INVALID, "tlno_gpu: nroots must be 1..9");
        if (fp32 < 0 || fp32 > 2 || (fp32 == 2 && nroots > 3))
            throw Error(TLNO_GPU_E_INVALID, "tlno_gpu: Rys evaluation mode out of range for nroots");
        for (int i = 0; i < n; ++i)
            if (!finite_bits(T[i]) || T[i] < 0.0) throw Error(TLNO_GPU_E_INVALID, "tlno_gpu: Rys argument must be finite and >= 0");
        set_device(device);
        ensure_device_tables();
        if (n == 0) return;
        DeviceBuffer dt, dr, dw;
        dt.alloc(sizeof(double) * n);
        dr.alloc(sizeof(double) * n * nroots);
        dw.alloc(sizeof(double) * n * nroots);
        TLNO_CUDA(cudaMemcpy(dt.ptr, T, sizeof(double) * n, cudaMemcpyHostToDevice));
        launch_rys_test(dt.as<double>(), n, nroots, fp32, dr.as<double>(), dw.as<double>(), 0);
        TLNO_CUDA(cudaMemcpy(roots, dr.ptr, sizeof(double) * n * nroots, cudaMemcpyDeviceToHost));
        TLNO_CUDA(cudaMemcpy(weights, dw.ptr, sizeof(double) * n * nroots, cudaMemcpyDeviceToHost));
    });
}

int tlno_gpu_fma_peak(int device, int fp32, double* tflops) {
    return guarded([&] {
        if (!tflops) throw Error(TLNO_GPU_E_INVALID, "tlno_gpu: null argument");
        set_device(device);
        *tflops = measure_fma_peak(fp32 != 0);
    });
}

int tlno_gpu_jk_graph_capture(tlno_gpu_context* ctx, const double* d_density, double* d_J, double* d_K, int flags) {
    return guarded([&] {
        if (!ctx || !d_density || !d_J || !d_K) throw Error(TLNO_GPU_E_INVALID, "tlno_gpu: null argument");
        if (!ctx->plan) throw Error(TLNO_GPU_E_STATE, "tlno_gpu: no plan; call tlno_gpu_plan first");
        TLNO_CUDA(cudaSetDevice(ctx->device));
        const int M = ctx->basis.n_sph;
        const long long n = static_cast<long long>(M) * M;
        ensure_work(ctx->w, 1);
        if (ctx->graph_exec) { cudaGraphExecDestroy(ctx->graph_exec); ctx->graph_exec = nullptr; }
        if (ctx->graph) { cudaGraphDestroy(ctx->graph); ctx->graph = nullptr; }
        const bool want_j = (flags & (TLNO_GPU_WANT_J | TLNO_GPU_WANT_G)) || !(flags & TLNO_GPU_WANT_K);
        const bool want_k = (flags & (TLNO_GPU_WANT_K | TLNO_GPU_WANT_G)) || !(flags & TLNO_GPU_WANT_J);
        float* d32 = nullptr;
        if (flags & TLNO_GPU_MIXED) {  // allocated before the capture
            ctx->w.D32.alloc(sizeof(float) * n);
            d32 = ctx->w.D32.as<float>();
        }
        validate_build_combination(ctx->screening);
        if (ctx->screening.density_threshold > 0.0) ensure_density_tables(*ctx->plan);
        const BuildSpec spec = spec_from(ctx->screening, want_j, want_k, flags & TLNO_GPU_MIXED,
                                         (flags & TLNO_GPU_WANT_G) != 0);
        TLNO_CUDA(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
        try {
            enqueue_jk(*ctx->plan, ctx->tune, spec, d_density, d_J, d_K, n, M, ctx->w.dmax.as<double>(), d32,
                       ctx->stream, &ctx->fan);
        } catch (...) {
            cudaGraph_t g = nullptr;
            cudaStreamEndCapture(ctx->stream, &g);
            if (g) cudaGraphDestroy(g);
            throw;
        }
        TLNO_CUDA(cudaStreamEndCapture(ctx->stream, &ctx->graph));
        TLNO_CUDA(cudaGraphInstantiate(&ctx->graph_exec, ctx->graph, 0));
    });
}

int tlno_gpu_jk_graph_launch(tlno_gpu_context* ctx) {
    return guarded([&] {
        if (!ctx || !ctx->graph_exec) throw Error(TLNO_GPU_E_STATE, "tlno_gpu: no captured graph");
        TLNO_CUDA(cudaSetDevice(ctx->device));
        TLNO_CUDA(cudaGraphLaunch(ctx->graph_exec, ctx->stream));
    });
}

int tlno_gpu_synchronize(tlno_gpu_context* ctx) {
    return guarded([&] {
        if (!ctx) throw Error(TLNO_GPU_E_INVALID, "tlno_gpu: null context");
        TLNO_CUDA(cudaSetDevice(ctx->device));
        TLNO_CUDA(cudaStreamSynchronize(ctx->stream));
    });
}

void* tlno_gpu_stream(tlno_gpu_context* ctx) { return ctx ? static_cast<void*>(ctx->stream) : nullptr; }

int tlno_gpu_set_tuning(tlno_gpu_context* ctx, const tlno_gpu_tuning* t) {
    return guarded([&] {
        if (!ctx || !t) throw Error(TLNO_GPU_E_INVALID, "tlno_gpu: null argument");
        if (t->generic_bk < 1 || t->generic_bk > 4096 || t->generic_warps < 0 || t->generic_warps > 8 ||
            t->grid_mult < 1 || t->grid_mult > 64 || t->streams < 1 || t->streams > 4)
            throw Error(TLNO_GPU_E_INVALID, "tlno_gpu: tuning value out of range");
        ctx->tune.streams = t->streams;
        ctx->tune.generic_bk = t->generic_bk;
        ctx->tune.generic_warps = t->generic_warps;
        ctx->tune.grid_mult = t->grid_mult;
    });
}

int tlno_gpu_set_combo_generic(tlno_gpu_context* ctx, int combo_id, int force_generic) {
    return guarded([&] {
        if (!ctx || combo_id < 0 || combo_id >= 256) throw Error(TLNO_GPU_E_INVALID, "tlno_gpu: bad combo id");
        ctx->tune.force_generic[combo_id] = force_generic ? 1 : 0;
    });
}

int tlno_gpu_plan_combos(const tlno_gpu_context* ctx, int max_n, int* ints, double* dbl) {
    int count = 0;
    const int rc = guarded([&] {
        if (!ctx || !ctx->plan) throw Error(TLNO_GPU_E_STATE, "tlno_gpu: no plan");
        for (const ComboSchedule& cs : ctx->plan->combos) {
            if (count < max_n) {
                int* o = ints + 8 * count;
                o[0] = cs.X; o[1] = cs.Y; o[2] = cs.la; o[3] = cs.lb; o[4] = cs.lc; o[5] = cs.ld;
                o[6] = cs.fast ? 1 : 0; o[7] = cs.n_tiles;
                dbl[3 * count] = static_cast<double>(cs.quartets);
                dbl[3 * count + 1] = static_cast<double>(cs.prim_quartets);
                dbl[3 * count + 2] = cs.flops;
            }
            ++count;
        }
    });
    return rc == TLNO_GPU_OK ? count : rc;
}

int tlno_gpu_time_combo(tlno_gpu_context* ctx, int combo_index, int mode, int reps, double* ms) {
    const int fp32 = mode & 1;
    return guarded([&] {
        if (!ctx || !ctx->plan || !ms) throw Error(TLNO_GPU_E_STATE, "tlno_gpu: no plan");
        Plan2e& plan = *ctx->plan;
        if (combo_index < 0 || combo_index >= static_cast<int>(plan.combos.size()))
            throw Error(TLNO_GPU_E_INVALID, "tlno_gpu: combo index out of range");
        TLNO_CUDA(cudaSetDevice(ctx->device));
        cudaStream_t s = ctx->stream;
        const int M = ctx->basis.n_sph;
        const long long n = static_cast<long long>(M) * M;
        ensure_work(ctx->w, n);
        ComboSchedule& cs = plan.combos[combo_index];
        dev::ClassLaunch cl{};
        cl.la = cs.la; cl.lb = cs.lb; cl.lc = cs.lc; cl.ld = cs.ld;
        cl.same = cs.X == cs.Y;
        cl.bb = cs.bb; cl.bk = cs.bk;
        cl.blocks = cs.d_blocks.as<dev::BlockDesc>();
        cl.bra_list = cs.d_bra_list.as<int>();
        cl.tile_prefix = cs.d_prefix.as<int>();
        cl.n_blocks = static_cast<int>(cs.blocks.size());
        cl.tile_begin = 0;
        cl.tile_end = cs.n_tiles;
        cl.tau = plan.tau;
        cl.chunk = cs.chunk;
        cl.dens = ctx->w.D.as<double>();
        ctx->w.D32.alloc(sizeof(float) * n);
        cl.dens32 = ctx->w.D32.as<float>();
        cl.J = ctx->w.J.as<double>();
        cl.K = ctx->w.K.as<double>();
        cl.M = M;
        cl.want_j = (mode & 2) ? 0 : 1;
        cl.want_k = (mode & 4) ? 0 : 1;
        int sms = 0;
        TLNO_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
        const int grid = sms * ctx->tune.grid_mult;
        cudaEvent_t e0, e1;
        TLNO_CUDA(cudaEventCreate(&e0));
        TLNO_CUDA(cudaEventCreate(&e1));
        const dev::PlanView pv = plan.view();
        cl.counter = plan.d_counters.as<int>() + 2 * combo_index;
        auto run = [&] {
            TLNO_CUDA(cudaMemsetAsync(cl.counter, 0, sizeof(int), s));
            if (cs.fast) launch_eri_jk_fast(pv, cl, fp32 != 0, grid, s);
            else launch_eri_jk_generic(pv, cl, fp32 != 0, ctx->tune.generic_warps, grid, s);
        };
        run();
        TLNO_CUDA(cudaEventRecord(e0, s));
        for (int r = 0; r < std::max(reps, 1); ++r) run();
        TLNO_CUDA(cudaEventRecord(e1, s));
        TLNO_CUDA(cudaEventSynchronize(e1));
        float t = 0.f;
        TLNO_CUDA(cudaEventElapsedTime(&t, e0, e1));
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        *ms = t / std::max(reps, 1);
    });
}

int tlno_gpu_set_class_tuning(tlno_gpu_context* ctx, int combo_index, double mixed_scale, int tile_chunk) {
    return guarded([&] {
        if (!ctx || !ctx->plan) throw Error(TLNO_GPU_E_STATE, "tlno_gpu: no plan");
        if (combo_index < 0 || combo_index >= static_cast<int>(ctx->plan->combos.size()))
            throw Error(TLNO_GPU_E_INVALID, "tlno_gpu: combo index out of range");
        if (!finite_bits(mixed_scale) || !(mixed_scale >= 0.0) || tile_chunk < 0 || tile_chunk > 64)
            throw Error(TLNO_GPU_E_INVALID, "tlno_gpu: class tuning value out of range");
        ctx->plan->combos[combo_index].mix_scale = mixed_scale;
        ctx->plan->combos[combo_index].chunk = tile_chunk;
    });
}

int tlno_gpu_class_jk(tlno_gpu_context* ctx, int combo_index, const double* d_density, double* d_J, double* d_K,
                      int flags, double* ms) {
    return guarded([&] {
        if (!ctx || !ctx->plan || !d_density || !d_J || !d_K) throw Error(TLNO_GPU_E_STATE, "tlno_gpu: no plan");
        Plan2e& plan = *ctx->plan;
        if (combo_index < 0 || combo_index >= static_cast<int>(plan.combos.size()))
            throw Error(TLNO_GPU_E_INVALID, "tlno_gpu: combo index out of range");
        TLNO_CUDA(cudaSetDevice(ctx->device));
        cudaStream_t s = ctx->stream;
        const int M = ctx->basis.n_sph;
        const long long n = static_cast<long long>(M) * M;
        ensure_work(ctx->w, 1);
        const bool mixed = flags & TLNO_GPU_MIXED;
        float* d32 = nullptr;
        if (mixed) {
            ctx->w.D32.alloc(sizeof(float) * n);
            d32 = ctx->w.D32.as<float>();
        }
        TLNO_CUDA(cudaMemsetAsync(d_J, 0, sizeof(double) * n, s));
        TLNO_CUDA(cudaMemsetAsync(d_K, 0, sizeof(double) * n, s));
        TLNO_CUDA(cudaMemsetAsync(plan.d_counters.ptr, 0, sizeof(int) * 2 * plan.combos.size(), s));
        if (mixed) launch_absmax_f32(d_density, n, ctx->w.dmax.as<double>(), d32, s);
        ComboSchedule& cs = plan.combos[combo_index];
        dev::ClassLaunch cl{};
        cl.la = cs.la; cl.lb = cs.lb; cl.lc = cs.lc; cl.ld = cs.ld;
        cl.same = (cs.X == cs.Y);
        cl.bb = cs.bb; cl.bk = cs.bk;
        cl.blocks = cs.d_blocks.as<dev::BlockDesc>();
        cl.bra_list = cs.d_bra_list.as<int>();
        cl.tile_prefix = cs.d_prefix.as<int>();
        cl.n_blocks = static_cast<int>(cs.blocks.size());
        cl.tile_begin = 0;
        cl.tile_end = cs.n_tiles;
        cl.tau = plan.tau;
        cl.tau_mix = ctx->screening.mixed_threshold * cs.mix_scale;
        cl.chunk = cs.chunk;
        cl.dmax = ctx->w.dmax.as<double>();
        cl.dens = d_density;
        cl.dens32 = d32;
        cl.J = d_J;
        cl.K = d_K;
        cl.M = M;
        cl.want_j = 1;
        cl.want_k = 1;
        int sms = 0;
        TLNO_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
        const dev::PlanView pv = plan.view();
        cudaEvent_t e0, e1;
        TLNO_CUDA(cudaEventCreate(&e0));
        TLNO_CUDA(cudaEventCreate(&e1));
        TLNO_CUDA(cudaEventRecord(e0, s));
        const bool split = mixed && cs.mix_scale > 0.0;
        for (int pass = 0; pass < (split ? 2 : 1); ++pass) {
            cl.prec_mode = split ? pass + 1 : 0;
            cl.counter = plan.d_counters.as<int>() + 2 * combo_index + pass;
            const bool fp32 = split && pass == 1;
            if (cs.fast)
                launch_eri_jk_fast(pv, cl, fp32, sms * ctx->tune.grid_mult, s);
            else
                launch_eri_jk_generic(pv, cl, fp32, ctx->tune.generic_warps, sms * ctx->tune.grid_mult, s);
        }
        TLNO_CUDA(cudaEventRecord(e1, s));
        TLNO_CUDA(cudaEventSynchronize(e1));
        float t = 0.f;
        TLNO_CUDA(cudaEventElapsedTime(&t, e0, e1));
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (ms) *ms = t;
    });
}

// ---------------- batch ----------------

int tlno_gpu_batch_create(int n_mol, tlno_gpu_context* const* ctxs, const tlno_gpu_screening* options,
                          tlno_gpu_batch** out) {
    return guarded([&] {
        if (!out || n_mol <= 0 || !ctxs) throw Error(TLNO_GPU_E_INVALID, "tlno_gpu: bad batch arguments");
        *out = nullptr;
        tlno_gpu_screening o = options ? *options : tlno_gpu_screening{1e-12, 0, 0, 0, 1e-9};
        validate_screening(o);
        auto b = std::make_unique<tlno_gpu_batch>();
        b->device = ctxs[0]->device;
        b->screening = o;
        b->tune = ctxs[0]->tune;
        set_device(b->device);
        ensure_device_tables();
        TLNO_CUDA(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
        std::vector<MolPairs> mps;
        for (int m = 0; m < n_mol; ++m) {
            if (!ctxs[m] || ctxs[m]->device != b->device)
                throw Error(TLNO_GPU_E_INVALID, "tlno_gpu: batch contexts must share one device");
            b->bases.push_back(ctxs[m]->basis);
        }
        for (int m = 0; m < n_mol; ++m)
            mps.push_back(build_mol_pairs(b->bases[m], o.integral_threshold, b->stream, o.decay_threshold));
        std::vector<const Basis*> bp;
        for (auto& x : b->bases) bp.push_back(&x);
        build_plan(b->plan, bp, std::move(mps), o.decay_threshold > 0.0 ? o.decay_threshold : o.integral_threshold,
                   b->tune, b->stream);
        b->plan.decay_metric = o.decay_threshold > 0.0;
        b->total = b->plan.mol_mat_off.back();
        *out = b.release();
    });
}

void tlno_gpu_batch_destroy(tlno_gpu_batch* b) { delete b; }

int tlno_gpu_batch_set_tuning(tlno_gpu_batch* b, const tlno_gpu_tuning* t) {
    return guarded([&] {
        if (!b || !t) throw Error(TLNO_GPU_E_INVALID, "tlno_gpu: null argument");
        if (t->generic_bk < 1 || t->generic_bk > 4096 || t->generic_warps < 0 || t->generic_warps > 8 ||
            t->grid_mult < 1 || t->grid_mult > 64 || t->streams < 1 || t->streams > 4)
            throw Error(TLNO_GPU_E_INVALID, "tlno_gpu: tuning value out of range");
        b->tune.generic_warps = t->generic_warps;
        b->tune.grid_mult = t->grid_mult;
        b->tune.streams = t->streams;
    });
}

long long tlno_gpu_batch_total_elements(const tlno_gpu_batch* b) { return b ? b->total : -1; }

int tlno_gpu_batch_offsets(const tlno_gpu_batch* b, long long* offsets) {
    return guarded([&] {
        if (!b || !offsets) throw Error(TLNO_GPU_E_INVALID, "tlno_gpu: null argument");
        std::copy(b->plan.mol_mat_off.begin(), b->plan.mol_mat_off.end(), offsets);
    });
}

int tlno_gpu_batch_profile(const tlno_gpu_batch* b, tlno_gpu_profile* out) {
    return guarded([&] {
        if (!b || !out) throw Error(TLNO_GPU_E_INVALID, "tlno_gpu: null argument");
        out->M = 0;
        for (int m : b->plan.mol_M) out->M += m;
        out->n_shells = b->plan.mol_shell_off.back();
        out->shell_pairs = b->plan.total_pairs;
        out->kept_pairs = b->plan.kept_pairs;
        out->quartets = b->plan.total_quartets;
        out->primitive_quartets = b->plan.total_prim_quartets;
        out->flops = b->plan.total_flops;
        out->n_class_launches = static_cast<int>(b->plan.combos.size());
    });
}

int tlno_gpu_batch_jk(tlno_gpu_batch* b, const double* density, double* J, double* K, int flags) {
    return guarded([&] {
        if (!b || !density || !J || !K) throw Error(TLNO_GPU_E_INVALID, "tlno_gpu: null argument");
        TLNO_CUDA(cudaSetDevice(b->device));
        cudaStream_t s = b->stream;
        ensure_work(b->w, b->total);
        const bool dev_ptrs = flags & TLNO_GPU_DEVICE_PTRS;
        const double* dD = density;
        if (!dev_ptrs) {
            if (!(flags & TLNO_GPU_NO_VALIDATE))
                for (int m = 0; m < b->plan.n_mol; ++m)
                    validate_density_host(density + b->plan.mol_mat_off[m], b->plan.mol_M[m]);
            TLNO_CUDA(cudaMemcpyAsync(b->w.D.ptr, density, sizeof(double) * b->total, cudaMemcpyHostToDevice, s));
            dD = b->w.D.as<double>();
        }
        double* dJ = dev_ptrs ? J : b->w.J.as<double>();
        double* dK = dev_ptrs ? K : b->w.K.as<double>();
        float* d32 = nullptr;
        if (flags & TLNO_GPU_MIXED) {
            b->w.D32.alloc(sizeof(float) * b->total);
            d32 = b->w.D32.as<float>();
        }
        validate_build_combination(b->screening);
        if (b->screening.density_threshold > 0.0) ensure_density_tables(b->plan);
        enqueue_jk(b->plan, b->tune, spec_from(b->screening, true, true, flags & TLNO_GPU_MIXED, false), dD, dJ, dK,
                   b->total, 0, b->w.dmax.as<double>(), d32, s, &b->fan);
        if (!dev_ptrs) {
            TLNO_CUDA(cudaMemcpyAsync(J, dJ, sizeof(double) * b->total, cudaMemcpyDeviceToHost, s));
            TLNO_CUDA(cudaMemcpyAsync(K, dK, sizeof(double) * b->total, cudaMemcpyDeviceToHost, s));
        }
        TLNO_CUDA(cudaStreamSynchronize(s));
    });
}

int tlno_gpu_batch_graph_capture(tlno_gpu_batch* b, const double* d_density, double* d_J, double* d_K, int flags) {
    return guarded([&] {
        if (!b || !d_density || !d_J || !d_K) throw Error(TLNO_GPU_E_INVALID, "tlno_gpu: null argument");
        TLNO_CUDA(cudaSetDevice(b->device));
        ensure_work(b->w, 1);
        if (b->graph_exec) { cudaGraphExecDestroy(b->graph_exec); b->graph_exec = nullptr; }
        if (b->graph) { cudaGraphDestroy(b->graph); b->graph = nullptr; }
        float* d32 = nullptr;
        if (flags & TLNO_GPU_MIXED) {  // allocated before the capture
            b->w.D32.alloc(sizeof(float) * b->total);
            d32 = b->w.D32.as<float>();
        }
        validate_build_combination(b->screening);
        if (b->screening.density_threshold > 0.0) ensure_density_tables(b->plan);
        const BuildSpec spec = spec_from(b->screening, true, true, flags & TLNO_GPU_MIXED, false);
        TLNO_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        try {
            enqueue_jk(b->plan, b->tune, spec, d_density, d_J, d_K, b->total, 0, b->w.dmax.as<double>(), d32,
                       b->stream, &b->fan);
        } catch (...) {
            cudaGraph_t g = nullptr;
            cudaStreamEndCapture(b->stream, &g);
            if (g) cudaGraphDestroy(g);
            throw;
        }
        TLNO_CUDA(cudaStreamEndCapture(b->stream, &b->graph));
        TLNO_CUDA(cudaGraphInstantiate(&b->graph_exec, b->graph, 0));
    });
}

int tlno_gpu_batch_graph_launch(tlno_gpu_batch* b) {
    return guarded([&] {
        if (!b || !b->graph_exec) throw Error(TLNO_GPU_E_STATE, "tlno_gpu: no captured graph");
        TLNO_CUDA(cudaSetDevice(b->device));
        TLNO_CUDA(cudaGraphLaunch(b->graph_exec, b->stream));
    });
}

int tlno_gpu_batch_synchronize(tlno_gpu_batch* b) {
    return guarded([&] {
        if (!b) throw Error(TLNO_GPU_E_INVALID, "tlno_gpu: null batch");
        TLNO_CUDA(cudaSetDevice(b->device));
        TLNO_CUDA(cudaStreamSynchronize(b->stream));
    });
}

void* tlno_gpu_batch_stream(tlno_gpu_batch* b) { return b ? static_cast<void*>(b->stream) : nullptr; }

}  // extern "C"
