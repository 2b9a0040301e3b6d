// Two-electron plan: Schwarz-screened shell pairs sorted by (La, Lb) class
// and bound, device-resident pair/primitive data and the quartet-class
// schedules; one-electron pair list.
#pragma once

#include <array>
#include <vector>

#include "engine.hpp"
#include "launch_types.hpp"

namespace tlno_gpu {

// Largest pair-projector table a plan keeps on the device; above it the
// generic classes run the warp-per-quartet kernel, which builds projectors
// per quartet.
constexpr long long kMaxProjectorBytes = 8LL << 30;

struct Tuning {
    int generic_bk = 64;    // ket pairs per tile of the warp-per-quartet kernel
    int generic_warps = 0;  // 0 = from shared-memory budget
    int grid_mult = 8;      // CTAs per SM for persistent launches
    int streams = 1;        // streams the class launches of a build spread over
    std::array<int, 256> force_generic{};  // per class combo: 1 = never use the fast kernel
};

struct ComboSchedule {
    int X = 0, Y = 0;            // pair classes, X >= Y
    int la = 0, lb = 0, lc = 0, ld = 0;
    bool fast = false;
    int bb = 1, bk = 16;
    // per-class tuning: split threshold multiplier of the mixed path and
    // tiles per dynamic-schedule fetch (0 = kernel default)
    double mix_scale = 1.0;
    int chunk = 0;
    std::vector<dev::BlockDesc> blocks;
    std::vector<int> prefix;
    std::vector<int> bra_list;
    DeviceBuffer d_blocks, d_prefix, d_bra_list;
    int n_tiles = 0;
    long long quartets = 0;       // surviving contracted quartets
    long long prim_quartets = 0;  // surviving primitive quartets
    double flops = 0.0;           // algorithmic flop model
};

// Pair data of one molecule (host), before merging into a device plan.
struct MolPairs {
    std::vector<int> A, B, nprim, cls;
    std::vector<double> Q;          // sorted order
    std::array<int, kMaxPairClasses> cls_begin{}, cls_count{};
    std::vector<double> Q_canonical;  // per canonical pair i*(i+1)/2+j
    double Qmax = 0.0;
};

class Plan2e {
public:
    // Device plan over one or more molecules (batch).
    double tau = 1e-12;
    int n_mol = 0;
    std::vector<int> mol_shell_off;   // global shell offset per molecule
    std::vector<int> mol_M;
    std::vector<long long> mol_mat_off;
    std::vector<MolPairs> mol_pairs;
    // Global sorted pair arrays (molecule-major, class, Q descending).
    std::vector<int> pair_A, pair_B, pair_nprim, pair_prim_off, pair_mol;
    std::vector<double> pair_Q;
    std::vector<ComboSchedule> combos;
    DeviceBuffer d_counters;  // dynamic-schedule counters, 2 per combo (FP64 and FP32 pass)
    DeviceBuffer d_shell_xyz, d_shell_L, d_shell_sph;
    DeviceBuffer d_pair_A, d_pair_B, d_pair_prim_off, d_pair_nprim, d_pair_Q, d_pair_mol;
    DeviceBuffer d_prim, d_prim32, d_mol_mat_off, d_mol_M;
    // Primitive FASTSCHWARZ estimate per primitive pair (prim order).
    DeviceBuffer d_prim_fs;
    // Density-screen tables: per molecule shell offset and count, offsets of
    // the ns x ns block tables, the tables and max |D| (allocated on first
    // use of density screening).
    std::vector<int> mol_ns;
    std::vector<long long> rho_off;
    DeviceBuffer d_mol_shell_off, d_mol_ns, d_rho_off, d_rho_blk, d_rho_max;
    long long max_ns2 = 0;
    // Shell-level metric of this plan: false = Schwarz bounds, true = the
    // heuristic decay indicator (integral_threshold must then be 0).
    bool decay_metric = false;
    // Pair projectors (HRR + spherical maps) of the pair classes the generic
    // class combinations use: per pair its offset into d_proj or -1.
    std::vector<long long> proj_off;
    DeviceBuffer d_proj, d_proj_off;
    long long proj_words = 0;
    bool proj_ready = false;
    long long total_quartets = 0, total_prim_quartets = 0;
    double total_flops = 0.0;
    long long total_pairs = 0, kept_pairs = 0;

    dev::PlanView view() const;
};

// Computes Schwarz bounds of every pair of a basis on the device and returns
// the sorted, screened pair list of that molecule.
// decay > 0 replaces the Schwarz bound by the reference's heuristic shell-pair
// decay indicator K_A K_B exp(-mu_min |AB|^2) (rys_engine.ipp:2205-2241) and
// screens the pair products against decay instead of tau.
MolPairs build_mol_pairs(const Basis& b, double tau, cudaStream_t s, double decay = 0.0);
// Allocates the density-screen tables of a plan (idempotent).
void ensure_density_tables(Plan2e& plan);

// Builds the device plan for a set of bases (one per molecule) with their
// already screened pair lists.
void build_plan(Plan2e& plan, const std::vector<const Basis*>& bases, std::vector<MolPairs>&& pairs,
                double tau, const Tuning& tune, cudaStream_t s);

// Primitive pair records of shells (A, B) with the reference's skip of zero
// coefficient products (rys_engine.ipp:2244-2279).
void primitive_pairs(const Basis& b, int A, int B, std::vector<dev::DPrimPair>& out);
int primitive_pair_count(const Basis& b, int A, int B);

// One-electron plan: kept shell pairs with the reference's group-pair decay
// screening (onee_matrices.cpp:96-216).
struct OneePlan {
    std::vector<dev::OneePair> pairs;
    std::vector<double> maxc;  // per primitive
    std::vector<double> nuc;   // x, y, z, Z of nonzero-charge nuclei
    double screen_thr = 0.0;
    DeviceBuffer d_pairs, d_maxc, d_nuc;
};
void build_onee_plan(OneePlan& p, const Basis& b, double decay_eps, double nuclear_eps);

}  // namespace tlno_gpu
