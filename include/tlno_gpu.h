/*
 * tlno_gpu.h -- C ABI of the B200 (sm_100a) integral engine.
 *
 * Drop-in boundary for the origo-tlno integral hot path.  Every entry point
 * replaces one C++ engine entry of the reference (cited per function, paths
 * relative to the reference repository) and keeps its argument meaning and
 * error contract: the reference throws std::runtime_error with an
 * "eri_ao_tensor_hgp:" prefix; here the same condition returns a negative
 * status and tlno_gpu_last_error() returns the same message text.
 *
 * Conventions
 *   - Status: 0 = success, < 0 = failure (TLNO_GPU_E_*).
 *   - Matrices are M x M row-major doubles over spherical AOs, shell by
 *     shell in input order, 2L+1 functions per shell in PySCF order
 *     (p: x, y, z; l >= 2: m = -l..l), the reference's AO order
 *     (integrals/one_electron/onee_matrices.cpp:459-484,
 *      integrals/two_electron/rys/rys_engine.ipp:2362-2383).
 *   - Buffers are host memory unless the call takes TLNO_GPU_DEVICE_PTRS,
 *     in which case every matrix pointer is CUDA device memory of the
 *     context's device.
 *   - One context = one basis, one CUDA device, one stream; a context is not
 *     thread-safe.  There is no CPU fallback: without a usable CUDA device
 *     every compute call fails with TLNO_GPU_E_CUDA.
 */
#ifndef TLNO_GPU_H
#define TLNO_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

#define TLNO_GPU_OK 0
#define TLNO_GPU_E_INVALID (-1)   /* invalid argument or input data        */
#define TLNO_GPU_E_CUDA (-2)      /* CUDA runtime error or no device       */
#define TLNO_GPU_E_STATE (-3)     /* call out of order (e.g. no plan yet)  */
#define TLNO_GPU_E_DEVICE (-4)    /* device-side status word reported fault */

/* flags */
#define TLNO_GPU_DEVICE_PTRS 0x1  /* matrix pointers are device memory       */
#define TLNO_GPU_WANT_J 0x2
#define TLNO_GPU_WANT_K 0x4
#define TLNO_GPU_WANT_G 0x8       /* G = J - K/2 (needs J and K internally)  */
#define TLNO_GPU_MIXED 0x10       /* mixed FP32/FP64 evaluation              */
#define TLNO_GPU_NO_VALIDATE 0x20 /* skip the density validation pass        */

typedef struct tlno_gpu_context tlno_gpu_context;

/* Screening options; field meaning of the reference's
 * fock::ScreeningOptions (integrals/two_electron/fock/jk_direct.hpp:18-24,
 * twoe_integrals.hpp:43-66) plus the mixed-precision split threshold.
 *   integral_threshold: Schwarz, keep shell quartets with Q_ab Q_cd >= tau.
 *   primitive_fastschwarz_threshold t: drop primitive quartets whose Simint
 *     FASTSCHWARZ estimate product is below t^2 (classes up to f); the
 *     reference drops a SIMD packet of primitive quartets only when all of
 *     its lanes fail, this engine drops each failing primitive quartet.
 *   decay_threshold: the heuristic shell-pair decay indicator
 *     K_A K_B exp(-mu |AB|^2) replaces the Schwarz bound as the pair metric;
 *     the reference's specialised route requires integral_threshold == 0
 *     with it, and so does this engine (same error text).
 *   density_threshold: CVHF density screen, q * max(4 max(rho_ab, rho_cd),
 *     max(rho_ac, rho_ad, rho_bc, rho_bd)) >= threshold with rho the
 *     shell-block maxima of |D| and the raised cutoff
 *     q >= max(tau, threshold / (4 max|D|)) (direct_build.ipp:122-251); J
 *     uses the Coulomb cap, K the exchange cap (with threshold / max|D|), G
 *     the larger of the two, as build_coulomb_j / build_exchange_k /
 *     build_rhf_g do.  Cannot be combined with decay_threshold. */
typedef struct {
    double integral_threshold;
    double primitive_fastschwarz_threshold;
    double decay_threshold;
    double density_threshold;
    double mixed_threshold;                 /* FP32 when Q_ab Q_cd max|D| < this */
} tlno_gpu_screening;

/* Plan statistics (the reference's EriPackedPlanProfile counterpart,
 * integrals/two_electron/twoe_integrals.hpp:166-187). */
typedef struct {
    int M;
    int n_shells;
    long long shell_pairs;          /* all canonical shell pairs            */
    long long kept_pairs;           /* pairs that can pass the Schwarz gate */
    long long quartets;             /* surviving unique contracted quartets */
    long long primitive_quartets;   /* surviving primitive quartets         */
    double flops;                   /* algorithmic flop model per J/K build */
    int n_class_launches;
} tlno_gpu_profile;

/* Last error message of the calling thread (empty string if none). */
const char* tlno_gpu_last_error(void);
/* ABI version (major * 10000 + minor * 100 + patch). */
int tlno_gpu_version(void);
/* Number of CUDA devices visible (0 when none). */
int tlno_gpu_device_count(int* count);

/* Create a context from contracted shells with RAW contraction coefficients;
 * every Cartesian component is normalised as the reference's make_shell does
 * (core/shell/shell_contract.cpp:41-48, core/basis/cartesian_shells.hpp:61-74).
 * centers: 3 per shell (bohr); L: 0..4; nprim: >= 1; exps/coefs: packed per
 * shell.  Z / atom_xyz: nuclear charges and centres for the attraction
 * integrals.  Replaces the std::vector<Shell> construction that feeds
 * build_one_electron_plan (onee_matrices.hpp:41) and build_direct_plan
 * (jk_direct.hpp:46). */
int tlno_gpu_create(int n_shells, const double* centers, const int* L, const int* nprim,
                    const double* exps, const double* coefs, int natom, const int* Z,
                    const double* atom_xyz, int device, tlno_gpu_context** out);

/* Create a context from per-Cartesian-component records that are already
 * normalised -- the reference's std::vector<core::basis::Shell> layout
 * (core/basis/types.hpp:30-35): centers 3 per component, ang 3 per
 * component, nprim per component, exps/coefs packed.  Components are grouped
 * into shells as the reference groups them (rys_engine.ipp:1928-2060). */
int tlno_gpu_create_from_components(int n_components, const double* centers, const int* ang,
                                    const int* nprim, const double* exps, const double* coefs,
                                    int natom, const int* Z, const double* atom_xyz, int device,
                                    tlno_gpu_context** out);

void tlno_gpu_destroy(tlno_gpu_context* ctx);

/* Spherical AO count M and shell count. */
int tlno_gpu_n_sph(const tlno_gpu_context* ctx);
int tlno_gpu_n_shells(const tlno_gpu_context* ctx);

/* Build the two-electron plan: Schwarz bounds on the device, class-sorted
 * screened pairs, quartet schedules.  Replaces fock::build_direct_plan
 * (integrals/two_electron/fock/jk_direct.hpp:46-48) and
 * build_eri_packed_plan_for_G_rys (twoe_integrals.hpp:202-204). */
int tlno_gpu_plan(tlno_gpu_context* ctx, const tlno_gpu_screening* options);
int tlno_gpu_plan_profile(const tlno_gpu_context* ctx, tlno_gpu_profile* out);

/* Coulomb / exchange build for a real symmetric density D (M x M).
 * flags: TLNO_GPU_WANT_J / _K / _G select outputs (null pointers allowed for
 * unselected ones), TLNO_GPU_MIXED selects the mixed-precision path,
 * TLNO_GPU_DEVICE_PTRS device-resident buffers.  Replaces
 * fock::build_coulomb_j, fock::build_exchange_k and fock::build_rhf_g
 * (integrals/two_electron/fock/jk_direct.hpp:82-96): J[a,b] = sum_cd
 * (ab|cd) D[c,d], K[a,c] = sum_bd (ab|cd) D[b,d], G = J - K/2. */
int tlno_gpu_jk(tlno_gpu_context* ctx, const double* density, double* J, double* K, double* G,
                int flags);

/* tlno_gpu_jk with the build-time screening options of the reference's
 * calls build_coulomb_j(plan, density, options) and its siblings
 * (jk_direct.hpp:82-96), which take the options again at build time:
 * density and primitive FASTSCHWARZ screening apply to this build; an
 * integral_threshold or decay_threshold other than the plan's re-plans
 * first (the options become the context's).  With TLNO_GPU_WANT_G alone it
 * is also the compatibility entry build_jk_direct_for_G_rys(plan, density,
 * options) (fock/eri_direct_jk.hpp:36-39): G = J - K/2 under the fused
 * density predicate.  mixed_threshold keeps the context's value. */
int tlno_gpu_jk_with_options(tlno_gpu_context* ctx, const double* density, double* J, double* K,
                             double* G, int flags, const tlno_gpu_screening* options);

/* ERI checksum stream: the sum of every canonical unique spherical ERI
 * (ij|kl), i >= j, k >= l, ij >= kl over AO pair indices, whose shell
 * quartet passes the plan's shell-level screen -- the value
 * build_eri_packed_for_G_rys returns in streaming mode
 * (integrals/two_electron/twoe_integrals.hpp:114-119, rys_engine.ipp:
 * 269-274, 690-708), and the ERI-only throughput endpoint timed by
 * benchmarks/two_electron_engine/src/twoe_timing.cpp.  FP64.  Requires a
 * plan; *ms (may be null) receives the device time of the kernels. */
int tlno_gpu_eri_checksum(tlno_gpu_context* ctx, double* checksum, double* ms);

/* Incremental (dP) RHF G builds for SCF iterations: the reference's
 * EriDirectJKIncrementalState (integrals/two_electron/fock/
 * eri_direct_jk.hpp:41-135, direct_build.ipp:562-775).  The first density,
 * every forced rebuild and every exact_rebuild_interval-th changed density
 * rebuild G = J - K/2 from the full density with density screening off;
 * the updates between contract dP = D - D_prev under
 * delta_density_threshold (or first_delta_density_threshold for the first
 * changed update after a rebuild when use_first_delta_density_threshold is
 * set) and add dG to the cached G.  An unchanged density is skipped.
 * Strong guarantee: a failed update leaves density, G, cadence, counters
 * and diagnostics as they were.  D and G live on the context's device. */
typedef struct tlno_gpu_incremental tlno_gpu_incremental;
typedef struct {
    tlno_gpu_screening base_options;        /* density_threshold is forced to 0 */
    unsigned long long exact_rebuild_interval; /* >= 1 */
    double delta_density_threshold;
    int use_first_delta_density_threshold;
    double first_delta_density_threshold;
} tlno_gpu_incremental_options;
#define TLNO_GPU_UPDATE_EXACT 1
#define TLNO_GPU_UPDATE_INCREMENTAL 2
#define TLNO_GPU_UPDATE_SKIPPED 3
typedef struct {
    unsigned long long updates, exact_rebuilds, incremental_updates, skipped_updates;
    int last_status;                        /* 0 before the first update */
    int initialized;
    double last_max_abs_density_delta;
    double last_effective_density_threshold;
    unsigned long long updates_since_exact_rebuild;
} tlno_gpu_incremental_info;
/* The state keeps a plan of its own built from options->base_options. */
int tlno_gpu_incremental_create(tlno_gpu_context* ctx, const tlno_gpu_incremental_options* options,
                                tlno_gpu_incremental** out);
void tlno_gpu_incremental_destroy(tlno_gpu_incremental* st);
/* Returns TLNO_GPU_UPDATE_* (>= 1) or a negative status.  flags:
 * TLNO_GPU_DEVICE_PTRS (density on the device), TLNO_GPU_MIXED (mixed
 * precision builds). */
int tlno_gpu_incremental_update(tlno_gpu_incremental* st, const double* density, int force_exact_rebuild,
                                int flags);
/* Copies the cached G (or the cached density) to G (host, or device with
 * TLNO_GPU_DEVICE_PTRS). */
int tlno_gpu_incremental_g(const tlno_gpu_incremental* st, double* G, int flags);
int tlno_gpu_incremental_density(const tlno_gpu_incremental* st, double* D, int flags);
int tlno_gpu_incremental_info_get(const tlno_gpu_incremental* st, tlno_gpu_incremental_info* out);
/* Back to the just-created state (plan and options kept). */
int tlno_gpu_incremental_reset(tlno_gpu_incremental* st);
/* Testing hook for the strong guarantee: the next update fails with
 * TLNO_GPU_E_STATE at `stage` (1 = after validation, before the build;
 * 2 = after the build, before the commit); 0 clears it. */
int tlno_gpu_incremental_fail_next_update(tlno_gpu_incremental* st, int stage);

/* One-electron S, T, V (spherical, M x M).  screening != 0 applies the
 * reference's default screening (group-pair decay 1e-15, nuclear primitive
 * 1e-15 / sum|Z|); 0 disables it.  Replaces
 * evaluate_one_electron_matrices_sph_into / build_one_electron_spherical_matrices
 * (integrals/one_electron/onee_matrices.hpp:50, 63-66). */
int tlno_gpu_onee(tlno_gpu_context* ctx, double* S, double* T, double* V, int screening, int flags);
/* Screening knobs (onee_matrices.hpp:78-79, onee_integrals.hpp:187-188). */
int tlno_gpu_set_onee_thresholds(tlno_gpu_context* ctx, double group_pair_decay_eps,
                                 double nuclear_screen_eps);

/* Split threshold of the mixed-precision J/K path (quartets with
 * Q_ab Q_cd max|D| below it run in FP32), as ScreeningOptions.mixed_threshold
 * without re-planning; used by the split-threshold autotuner.  No reference
 * counterpart (the reference has no mixed-precision path).  A captured J/K
 * graph keeps the value of its capture: capture again after a change. */
int tlno_gpu_set_mixed_threshold(tlno_gpu_context* ctx, double mixed_threshold);

/* Contracted spherical ERI blocks (A B | C D) for n quartets of shell
 * indices (4 per quartet); block q is written at out + offsets[q] with layout
 * [(2La+1)(2Lb+1)] x [(2Lc+1)(2Ld+1)] row-major.  Host buffers.  The
 * per-quartet producer of the reference is compute_quartet_block_rys_impl
 * followed by the final pair projector (rys_engine.ipp:13754, 1844). */
int tlno_gpu_eri_blocks(tlno_gpu_context* ctx, int n_quartets, const int* shells4,
                        const long long* offsets, double* out);

/* The same ERI blocks as tlno_gpu_eri_blocks, without any device
 * allocation: no cudaMalloc, cudaFree or allocating library call.  The call
 * blocks until its copy and kernels have finished (it synchronises the
 * context's stream); work the caller queued on other streams that touches
 * d_out must be finished before the call.  For
 * callers that cannot allocate device memory -- code that works inside a
 * device-memory budget owned by another allocator (a framework's pool), on a
 * latency-critical path where an allocation may synchronise the device, or
 * that must not grow its device footprint after start-up.  No counterpart
 * in the reference (its engine is CPU-only).
 * d_out is caller-owned device memory of the context's device; block q is
 * written at d_out + offsets[q] (element offsets, host array); shells4 is a
 * host array.  Per-call scratch (pair tables, primitive pairs, quartet lists)
 * lives in one fixed 8 MiB device array that every device on which a
 * context is created holds until exit (context creation looks up its
 * address with cudaGetSymbolAddress, which loads it); a request needing more
 * fails with TLNO_GPU_E_INVALID and a message naming the sizes (split it).
 * All calls share the array: calls that overlap on the GPU (e.g. from two
 * host threads) race. */
int tlno_gpu_eri_blocks_noalloc(tlno_gpu_context* ctx, int n_quartets, const int* shells4,
                                const long long* offsets, double* d_out);

/* Schwarz bound per canonical shell pair i*(i+1)/2 + j (i >= j), as
 * get_rys_spherical_pair_schwarz_bounds().pair_group_max
 * (rys_engine.ipp:16165-16258).  Requires a plan.  Host buffer. */
int tlno_gpu_schwarz(const tlno_gpu_context* ctx, double* out);

/* Device Boys function F_0..F_maxn at n points (host buffers; out is
 * n x (maxn+1)).  Reference: core/math/general_math.hpp:6-22. */
int tlno_gpu_boys(int device, int n, int maxn, const double* x, double* out);
/* Device Rys roots (t^2) and weights for nroots at n arguments (host
 * buffers, n x nroots each).  Reference: rys_roots_weights
 * (rys_engine.ipp:3823-3838).  fp32 selects the evaluation path of the
 * kernels: 0 = FP64 tables (the reference's 0.01-grid interpolant),
 * 1 = FP32 tables, 2 = the FP32 interval polynomials of the mixed-precision
 * kernels (nroots <= 3). */
int tlno_gpu_rys(int device, int n, int nroots, const double* T, double* roots, double* weights,
                 int fp32);

/* Measured FP64 FMA throughput of the device (TFLOP/s, 2 flops per FMA)
 * from a dependent-chain DFMA kernel filling every SM; the roofline
 * denominator of the FP64 ERI kernels.  fp32 != 0 measures FFMA instead. */
int tlno_gpu_fma_peak(int device, int fp32, double* tflops);

/* CUDA graph of one J/K build on device buffers (TLNO_GPU_DEVICE_PTRS is
 * implied): capture once, replay per SCF step after updating D in place. */
int tlno_gpu_jk_graph_capture(tlno_gpu_context* ctx, const double* d_density, double* d_J,
                              double* d_K, int flags);
int tlno_gpu_jk_graph_launch(tlno_gpu_context* ctx);
/* Waits for the context's stream. */
int tlno_gpu_synchronize(tlno_gpu_context* ctx);
/* Raw CUDA stream of the context (cudaStream_t) for event timing. */
void* tlno_gpu_stream(tlno_gpu_context* ctx);

/* Batched J/K over many molecules in one work queue per class (the
 * reference has no batch API; its per-molecule equivalent is repeated
 * build_coulomb_j / build_exchange_k calls).  The batch context owns the
 * merged plan; densities, J and K are stacked M_m x M_m blocks in molecule
 * order (offsets returned by tlno_gpu_batch_offsets). */
typedef struct tlno_gpu_batch tlno_gpu_batch;
int tlno_gpu_batch_create(int n_mol, tlno_gpu_context* const* ctxs, const tlno_gpu_screening* options,
                          tlno_gpu_batch** out);
void tlno_gpu_batch_destroy(tlno_gpu_batch* b);
long long tlno_gpu_batch_total_elements(const tlno_gpu_batch* b);
int tlno_gpu_batch_offsets(const tlno_gpu_batch* b, long long* offsets);
int tlno_gpu_batch_profile(const tlno_gpu_batch* b, tlno_gpu_profile* out);
int tlno_gpu_batch_jk(tlno_gpu_batch* b, const double* density, double* J, double* K, int flags);
int tlno_gpu_batch_graph_capture(tlno_gpu_batch* b, const double* d_density, double* d_J, double* d_K,
                                 int flags);
int tlno_gpu_batch_graph_launch(tlno_gpu_batch* b);
int tlno_gpu_batch_synchronize(tlno_gpu_batch* b);
void* tlno_gpu_batch_stream(tlno_gpu_batch* b);

/* Tuning of the kernel schedule: generic-kernel ket tile, generic warps
 * per CTA (0 = the block-per-quartet generic kernel with the plan's pair
 * projectors, or, for a plan too large to keep them, the warp-per-quartet
 * kernel with warps from the shared-memory budget; 1..8 = the
 * warp-per-quartet kernel with that many warps), persistent grid multiplier
 * (the compile-time kernels size their grid from the occupancy calculator,
 * capped by grid_mult x SMs), and streams (1..4): the class launches of a
 * build spread over that many streams (parallel branches of a captured
 * graph), so that the tail of one class overlaps the next; 1 keeps them in
 * order on the context's stream.  A per-class-combination generic override
 * is set separately. */
typedef struct {
    int generic_bk;
    int generic_warps;
    int grid_mult;
    int streams;
} tlno_gpu_tuning;
int tlno_gpu_set_tuning(tlno_gpu_context* ctx, const tlno_gpu_tuning* t);
/* The same for a batch (its schedule keeps the ket tile of its plan). */
int tlno_gpu_batch_set_tuning(tlno_gpu_batch* b, const tlno_gpu_tuning* t);
int tlno_gpu_set_combo_generic(tlno_gpu_context* ctx, int combo_id, int force_generic);
/* Per class-combination statistics of the current plan: for i < n, writes
 * (X, Y, la, lb, lc, ld, fast, n_tiles) into ints[8*i] and
 * (quartets, prim_quartets, flops) into dbl[3*i]; returns the count. */
int tlno_gpu_plan_combos(const tlno_gpu_context* ctx, int max_n, int* ints, double* dbl);
/* Per-class tuning of the current plan (the per-class autotuner's knobs;
 * no reference counterpart): the split threshold of class combination
 * combo_index is mixed_threshold x mixed_scale (>= 0; 0 keeps the class in
 * FP64 in a mixed build: one launch, no FP32 pass), and its compile-time
 * kernel takes tile_chunk tiles of 32 ket pairs per fetch of its dynamic
 * schedule (1..64; 0 = the kernel's default of 4).  Re-planning resets
 * them.  A captured J/K graph keeps the values of its capture. */
int tlno_gpu_set_class_tuning(tlno_gpu_context* ctx, int combo_index, double mixed_scale, int tile_chunk);
/* J and K contributions of one class combination alone (device buffers,
 * J and K zeroed first, not symmetrised), FP64 or with TLNO_GPU_MIXED the
 * split of the class's tuning; *ms (may be null) receives the device time of
 * the class kernels.  For the per-class autotuner's error and time model. */
int tlno_gpu_class_jk(tlno_gpu_context* ctx, int combo_index, const double* d_density, double* d_J,
                      double* d_K, int flags, double* ms);
/* Time one class combination alone (ms per launch, CUDA events) for the
 * autotuner; runs on the context's stream with its device buffers.
 * mode bits: 1 = FP32 evaluation, 2 = skip the J digestion, 4 = skip the K
 * digestion (2|4 = ERI evaluation only). */
int tlno_gpu_time_combo(tlno_gpu_context* ctx, int combo_index, int mode, int reps, double* ms);

#ifdef __cplusplus
}
#endif

#endif /* TLNO_GPU_H */
