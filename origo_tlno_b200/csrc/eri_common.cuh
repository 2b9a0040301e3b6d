// Launch descriptors and J/K digestion shared by the ERI kernels.
#pragma once

#include "device_common.cuh"
#include "launch_types.hpp"

namespace tlno_gpu {
namespace dev {

enum Mode { kStore = 0, kSchwarz = 1, kJK = 2 };

// Bra-block index of a linear tile via binary search in the prefix array.
__device__ __forceinline__ int find_block(const int* prefix, int n_blocks, int tile) {
    int lo = 0, hi = n_blocks - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(prefix + mid) <= tile) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// Density (CVHF) screen of one quartet of global shells (A B | C D) of
// molecule `mol` with pair metric product q (the plan's Schwarz test already
// passed): whether its Coulomb (lj) and exchange (lk) contributions are kept.
// Same predicate as the reference (native_quartets.ipp:499-518,
// rys_engine.ipp:1126-1167) with the raised cutoff of direct_build.ipp:229-251.
__device__ __forceinline__ void density_live(const ClassLaunch& cl, const PlanView& pv, int mol, int A, int B,
                                             int C, int D, double q, bool& lj, bool& lk) {
    const DensityScreen& ds = cl.den;
    const int so = pv.mol_shell_off ? __ldg(pv.mol_shell_off + mol) : 0;
    const int n = pv.mol_ns ? __ldg(pv.mol_ns + mol) : 0;
    const double* blk = ds.rho_blk + (ds.rho_off ? __ldg(ds.rho_off + mol) : 0);
    const int a = A - so, b = B - so, c = C - so, d = D - so;
    const int ns = pv.mol_ns ? n : cl.M_shells;
    const double rab = __ldg(blk + (long long)a * ns + b), rcd = __ldg(blk + (long long)c * ns + d);
    const double coul = 4.0 * fmax(rab, rcd);
    const double rho = __ldg(ds.rho_max + mol);
    double tj = cl.tau, tk = cl.tau;
    if (rho > 0.0) {
        tj = fmax(cl.tau, ds.thr / (rho * 4.0));
        tk = fmax(cl.tau, ds.thr / rho);
    }
    const double exch = fmax(fmax(__ldg(blk + (long long)c * ns + a), __ldg(blk + (long long)d * ns + a)),
                             fmax(__ldg(blk + (long long)c * ns + b), __ldg(blk + (long long)d * ns + b)));
    if (ds.mode == 2) {
        lj = lk = (q >= tj) && (q * fmax(coul, exch) >= ds.thr);
    } else {
        lj = (q >= tj) && (q * coul >= ds.thr);
        lk = (q >= tk) && (q * exch >= ds.thr);
    }
}

// Canonical AO pair index of (i, j): max(i,j) (max(i,j)+1) / 2 + min(i,j).
__device__ __forceinline__ long long ao_pair_index(int i, int j) {
    const long long hi = i > j ? i : j, lo = i > j ? j : i;
    return hi * (hi + 1) / 2 + lo;
}

// Whether element (a0+sa, b0+sb | c0+sc, d0+sd) of quartet (AB|CD) belongs
// to the canonical unique set of the ERI stream: i >= j inside a shell pair
// with A == B, k >= l with C == D, and kl <= ij when bra and ket are the
// same shell pair (rys_engine.ipp:690-708).
__device__ __forceinline__ bool canonical_element(bool same_ab, bool same_cd, bool same_pair, int a0, int sa,
                                                  int b0, int sb, int c0, int sc, int d0, int sd) {
    if (same_ab && sb > sa) return false;
    if (same_cd && sd > sc) return false;
    if (same_pair && ao_pair_index(c0 + sc, d0 + sd) > ao_pair_index(a0 + sa, b0 + sb)) return false;
    return true;
}

// Smallest pair metric product that can pass the density screen of molecule
// `mol` (the raised cutoff), for whole-tile skips.
__device__ __forceinline__ double density_tau_min(const ClassLaunch& cl, int mol) {
    const double rho = __ldg(cl.den.rho_max + mol);
    return rho > 0.0 ? fmax(cl.tau, cl.den.thr / (rho * 4.0)) : cl.tau;
}

}  // namespace dev
}  // namespace tlno_gpu
