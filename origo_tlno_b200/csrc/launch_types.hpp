// Plain launch descriptors shared by the host engine and the device code
// (no device-only constructs, so host C++ translation units can include it).
#pragma once

namespace tlno_gpu {
namespace dev {

struct DPrimPair {
    double p, Px, Py, Pz, w, invp;
};

// FP32 copy for the mixed-precision kernels: P relative to the pair's first
// centre A, so that FP32 never subtracts two absolute coordinates.
struct FPrimPair {
    float p, PAx, PAy, PAz, w, invp;
};

// Device view of one plan (or of a batch of plans: every pair carries the
// AO offset of its molecule, so one launch can serve many molecules).
struct PlanView {
    const double* shell_xyz;      // 3 per shell
    const int* shell_L;
    const int* shell_sph;         // first spherical AO of the shell (molecule-local)
    const int* pair_A;            // oriented shells, L_A >= L_B
    const int* pair_B;
    const int* pair_prim_off;
    const int* pair_nprim;
    const double* pair_Q;         // Schwarz bound
    const int* pair_mol;          // molecule of the pair (batch), may be null
    const DPrimPair* prim;
    const FPrimPair* prim32;      // same records in FP32 (P relative to A), may be null
    // Per-molecule matrix bases (batch): density/J/K at base + M*M offsets.
    const long long* mol_mat_off; // element offset of the molecule's M x M block
    const int* mol_M;
    // Primitive FASTSCHWARZ estimate per primitive pair (same order as prim):
    // 24.7394... w^2 sqrt(1/p) (rys_engine.ipp:2264-2268); may be null.
    const double* prim_fs;
    // Per molecule: first global shell and shell count (density tables are
    // indexed by molecule-local shells); null for a single molecule.
    const int* mol_shell_off;
    const int* mol_ns;
    // HRR + spherical projector of each pair used by a generic class
    // combination: proj + proj_off[pair], stored transposed (column = the
    // Cartesian slice |a'| in [La, La+Lb], row = s_ab, rows contiguous);
    // null when the plan keeps none.
    const double* proj;
    const long long* proj_off;
};

// Density (CVHF) screen of one build (direct_build.ipp:122-251,
// native_quartets.ipp:499-518): a quartet of pair metric product q passes the
// Coulomb test when q >= max(tau, thr / (4 rho_max)) and
// q * 4 max(rho_ab, rho_cd) >= thr, the exchange test when
// q >= max(tau, thr / rho_max) and q * max(rho_ac, rho_ad, rho_bc, rho_bd) >= thr,
// the fused (G) test when q >= max(tau, thr / (4 rho_max)) and
// q * max(coulomb cap, exchange cap) >= thr.
struct DensityScreen {
    int mode;                     // 0 off; 1 J and K tested apart; 2 fused G test
    double thr;                   // density_threshold
    const double* rho_blk;        // per molecule ns x ns shell-block maxima of |D| (flat)
    const long long* rho_off;     // per molecule offset into rho_blk (null: single molecule)
    const double* rho_max;        // per molecule max |D|
};

// One block of a quartet-class schedule: `nbra` bra pairs (entries bra0 ..
// bra0+nbra-1 of the launch's bra list; for the compile-time kernels they
// share their first shell) against one segment of the ket class list of the
// same molecule (the kets of a segment share their primitive count).
struct BlockDesc {
    int bra0;      // first entry in ClassLaunch::bra_list
    int nbra;      // bras in this block
    int ket0;      // first pair of the ket segment (global sorted index)
    int nket;      // length of the segment
    int xbeg;      // first pair of the bra class list of this molecule
                   // (triangle test on the diagonal class: i = bra - xbeg)
    int koff;      // position of the segment inside the ket class list
};

// Quartet class and the schedule of one launch.
struct ClassLaunch {
    int la, lb, lc, ld;
    int same;                     // bra class == ket class (triangle j <= i)
    int bb, bk;                   // tile shape: bra pairs x ket pairs
    const BlockDesc* blocks;
    const int* bra_list;          // bra pair (global sorted index) per block entry
    const int* tile_prefix;       // per block: first tile index (n_blocks + 1)
    int n_blocks;
    int tile_begin, tile_end;     // tile range of this launch
    int* counter;                 // dynamic-schedule counter, zero at launch (compile-time kernels)
    int chunk;                    // tiles per counter fetch (0 = kernel default)
    double tau;                   // Schwarz threshold
    // Precision split: mode 0 = every quartet; 1 = quartets with
    // Q_ab Q_cd max|D| >= tau_mix only (FP64 part); 2 = the complement.
    int prec_mode;
    double tau_mix;
    const double* dmax;           // device scalar max|D| (per build)
    // Explicit quartet list (STORE / SCHWARZ modes): pair indices.
    const int* q_bra;
    const int* q_ket;
    int n_quartets;
    // Outputs.
    double* out;                  // STORE: blocks; SCHWARZ: Q per quartet
    const long long* out_off;     // STORE: element offset per quartet
    const double* dens;
    const float* dens32;          // FP32 copy of dens (FP32 kernels of a mixed build)
    double* J;
    double* K;
    int M;                        // single-molecule AO count (when no batch)
    int M_shells;                 // single-molecule shell count (when no batch)
    int want_j, want_k;
    unsigned int* status;         // device error word (0 = ok)
    DensityScreen den;
    double fs_thr2;               // primitive FASTSCHWARZ threshold squared (0 = off)
    // ERI checksum stream (J/K kernels with want_j = want_k = 0): the sum of
    // the canonical unique spherical ERIs of the launch is added here.
    double* checksum;
};

struct OneePair {
    int A, B;         // oriented shells, L_A >= L_B
    int do_st, do_v;
};

struct OneeLaunch {
    const double* shell_xyz;
    const int* shell_L;
    const int* shell_nprim;
    const int* shell_prim;
    const int* shell_sph;
    const double* exps;
    const double* c_radial;
    const double* maxc;        // per primitive: max |normalised coefficient| over the group
    const double* comp_coef;   // normalised coefficient per Cartesian component and primitive
    const int* comp_off;       // per shell: offset into comp_coef
    const OneePair* pairs;
    int n_pairs;
    const double* nuc;         // 4 per nucleus: x, y, z, Z (zero-charge nuclei removed)
    int n_nuc;
    double screen_thr;         // eps / sum|Z| (0 disables)
    int M;
    double* S;
    double* T;
    double* V;
};

}  // namespace dev
}  // namespace tlno_gpu
