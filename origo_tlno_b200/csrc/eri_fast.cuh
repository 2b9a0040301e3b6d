// Compile-time-class Rys ERI + J/K kernel for angular momenta up to d
// (thread per contracted quartet, the quartet's work sliced over TPQ warps).
//
// Tile: a group of TPQ warps takes one bra shell pair and 32 consecutive ket
// shell pairs of one primitive-count segment of the same class (one quartet
// per lane); a CTA holds BBQ independent groups, each pulling chunks of
// tiles from a launch counter.
//
// Phase 1 (registers): every thread of a quartet evaluates the primitive
// loop (Rys roots/weights, 2-D VRR) and accumulates its own slice of the
// contracted radial integrals (a0|c0): rows ia = g, g+TPQ, ... of the
// NAS x NCS block, g = warp index inside the group.  The slice is fixed at
// compile time, so the accumulators stay in registers; TPQ is the smallest
// power of two whose slice holds at most fast_acc_limit() accumulators.
// Phase 2: ket HRR and ket spherical projection of the owned rows, written
// to shared memory as (a0|cd)_sph rows.
// Phase 3: after a barrier, each warp takes a share of the ket columns
// (c,d)_sph, applies the bra HRR and projection and digests the finished
// (ab|cd) column into J and K (J[ab] warp-reduced, the rest FP64 atomics
// from per-thread partial sums).
//
// Arithmetic follows the reference's producer: contracted radial
// accumulation, contracted-space HRR, final pair projection
// (rys_engine.ipp:12585-13748, 3141-3362, 1801-1860) and the 8-fold J/K
// digestion (consumer_policies.ipp:87-221).
#pragma once

#include <type_traits>
#include <utility>

#include "eri_common.cuh"

namespace tlno_gpu {
namespace dev {

__host__ __device__ constexpr int ce_ncart(int L) { return (L + 1) * (L + 2) / 2; }
__host__ __device__ constexpr int ce_nsph(int L) { return 2 * L + 1; }
__host__ __device__ constexpr int ce_off(int L) { return L * (L + 1) * (L + 2) / 6; }
__host__ __device__ constexpr int ce_cum(int L) { return (L + 1) * (L + 2) * (L + 3) / 6; }
// Cartesian exponents of flat index f (reference order: lx = L..0, then
// ly = L-lx..0), in closed form so that they fold at compile time.
__host__ __device__ constexpr int ce_L(int f) {
    int L = 0;
    while (ce_cum(L) <= f) ++L;
    return L;
}
// dx = L - lx: the local index is dx(dx+1)/2 + lz.
__host__ __device__ constexpr int ce_dx(int f) {
    const int loc = f - ce_off(ce_L(f));
    int dx = 0;
    while ((dx + 1) * (dx + 2) / 2 <= loc) ++dx;
    return dx;
}
__host__ __device__ constexpr int ce_x(int f) { return ce_L(f) - ce_dx(f); }
__host__ __device__ constexpr int ce_z(int f) {
    const int dx = ce_dx(f);
    return f - ce_off(ce_L(f)) - dx * (dx + 1) / 2;
}
__host__ __device__ constexpr int ce_y(int f) { return ce_dx(f) - ce_z(f); }
__host__ __device__ constexpr int ce_flat(int x, int y, int z) {
    return ce_off(x + y + z) + (y + z) * (y + z + 1) / 2 + z;
}
static_assert(ce_x(ce_flat(2, 1, 0)) == 2 && ce_y(ce_flat(2, 1, 0)) == 1 && ce_z(ce_flat(0, 1, 3)) == 3 &&
                  ce_x(ce_flat(0, 0, 4)) == 0 && ce_z(ce_flat(1, 1, 1)) == 1,
              "Cartesian index round trip");

// Non-zero pattern of the Cartesian->spherical map (real solid harmonics,
// order m = -l..l; Cartesians xx, xy, xz, yy, yz, zz for d), so that the
// projection skips structural zeros at compile time.
__host__ __device__ constexpr bool c2s_nz(int L, int s, int c) {
    if (L <= 1) return s == c;
    if (L == 2) {
        return (s == 0 && c == 1) || (s == 1 && c == 4) || (s == 2 && (c == 0 || c == 3 || c == 5)) ||
               (s == 3 && c == 2) || (s == 4 && (c == 0 || c == 3));
    }
    return true;
}

constexpr int kTileChunk = 4;  // default tiles per dynamic-schedule fetch
constexpr int kBraGroup = 8;   // bras per block of the light classes
constexpr int kMaxCarried = 24;

// Radial accumulators per thread slice.  Every slice of a quartet repeats the
// primitive loop (roots, 2-D VRR) and is its own unrolled copy of the code,
// so fewer, wider slices win although they need more registers: 128
// (cfg4 (dp|pp): FP64 1108 -> 757 ms, FP32 934 -> 579 ms, with FP64 spills;
// cfg2's compile-time f classes: FP64 1639 -> 1126 ms, FP32 1474 -> 783 ms),
// except (dp|dp), which spills too much in FP64 (310 -> 391 ms) and keeps 64.
__host__ __device__ constexpr int fast_acc_limit(int la, int lb, int lc, int ld) {
    return (la == 2 && lb == 1 && lc == 2 && ld == 1) ? 64 : 128;
}

__host__ __device__ constexpr int fast_pick_tpq(int nas, int ncs, int acc) {
    int t = 1;
    while (t < 32 && ((nas + t - 1) / t) * ncs > acc) t *= 2;
    return t;
}

template <int LA, int LB, int LC, int LD>
struct FastShape {
    static constexpr int LAB = LA + LB, LCD = LC + LD;
    static constexpr int N = (LAB + LCD) / 2 + 1;
    static constexpr int KS = LCD + 1;
    static constexpr int GS = (LAB + 1) * KS;
    static constexpr int OFA = ce_off(LA), NAS = ce_cum(LAB) - OFA;
    static constexpr int OFC = ce_off(LC), NCS = ce_cum(LCD) - OFC;
    static constexpr int NCA = ce_ncart(LA), NCB = ce_ncart(LB);
    static constexpr int NCC = ce_ncart(LC), NCD = ce_ncart(LD);
    static constexpr int NSA = ce_nsph(LA), NSB = ce_nsph(LB);
    static constexpr int NSC = ce_nsph(LC), NSD = ce_nsph(LD);
    static constexpr int NSAB = NSA * NSB, NSCD = NSC * NSD;
    static constexpr int TPQ = fast_pick_tpq(NAS, NCS, fast_acc_limit(LA, LB, LC, LD));
    static constexpr int BBQ = TPQ >= 4 ? 1 : 4 / TPQ;
    static constexpr int WARPS = TPQ * BBQ;
    // Phase-3 work split: by ket spherical function c when there are enough
    // of them (K[ac], K[bc] complete inside one warp), else by column (c,d).
    static constexpr bool BY_SC = NSC >= TPQ;
    // Bras per schedule block, all with the same first shell A: a lane's
    // J[cd], K[ac] and K[ad] sums stay in registers across the block, which
    // divides those FP64 atomics by the block size.  Only for unsliced
    // classes whose carried sums are small.
    static constexpr int GB = (TPQ == 1 && NSA * (NSC + NSD) + NSCD <= kMaxCarried) ? kBraGroup : 1;
    static constexpr int LANE_STRIDE = (NAS * NSCD) | 1;  // odd: conflict-free FP64 rows
    static constexpr int SMEM_DOUBLES = TPQ == 1 ? 0 : BBQ * 32 * LANE_STRIDE;
    // Bra-group classes: per lane, the density values every bra of a block
    // shares (D[a,c], D[a,d], D[c,d]), gathered once per tile.
    static constexpr int PRE_VALS = GB > 1 ? NSA * NSC + NSA * NSD + NSCD : 0;
};

// Binomial C(n, k) for the small HRR exponents.
__host__ __device__ constexpr int ce_binom(int n, int k) {
    int num = 1, den = 1;
    for (int i = 0; i < k; ++i) { num *= n - i; den *= i + 1; }
    return num / den;
}

// Compile-time loop: f(integral_constant<int, 0>) ... f(integral_constant<int, N-1>),
// so that every index derived from the loop variable is a constant expression
// (register arrays stay in registers, no unroller/folding round trips).
template <typename F, int... Is>
__device__ __forceinline__ void sfor_seq(F&& f, std::integer_sequence<int, Is...>) {
    (f(std::integral_constant<int, Is>{}), ...);
}
template <int N, typename F>
__device__ __forceinline__ void sfor(F&& f) {
    if constexpr (N > 0) sfor_seq(f, std::make_integer_sequence<int, N>{});
}
#define TLNO_CI(x) decltype(x)::value

// HRR transfer coefficient C(B,U) X^(B-U).
template <int B, int U, typename T>
__device__ __forceinline__ T hrr_coef(T x) {
    constexpr int e = B - U;
    constexpr T c = T(ce_binom(B, U));
    if constexpr (e == 0) return T(1);
    else if constexpr (e == 1) return c * x;
    else if constexpr (e == 2) return c * (x * x);
    else if constexpr (e == 3) return c * (x * x * x);
    else return c * ((x * x) * (x * x));
}

// Spherical element (S1, S2) of a shell pair (L1 >= L2) from the rows
// (l1+u, 0) of its Cartesian range, l1 + u in [L1, L1+L2] (flat index minus
// OF): horizontal transfer (a,b) = sum_u C(b,u) X^(b-u) (a+u, 0) with
// X = centre1 - centre2, then the Cartesian->spherical projection with the
// angular normalisation folded in.  src(integral_constant<int, f>) returns
// row f.
template <typename T, int L1, int L2, int S1, int S2, int OF, typename Src>
__device__ __forceinline__ T pair_transfer(const T* X, Src&& src) {
    T out = T(0);
    sfor<ce_ncart(L1)>([&](auto C1) {
        constexpr int c1 = TLNO_CI(C1);
        if constexpr (c2s_nz(L1, S1, c1)) {
            constexpr int f1 = ce_off(L1) + c1;
            T row = T(0);
            sfor<ce_ncart(L2)>([&](auto C2) {
                constexpr int c2 = TLNO_CI(C2);
                if constexpr (c2s_nz(L2, S2, c2)) {
                    constexpr int f2 = ce_off(L2) + c2;
                    constexpr int bx = ce_x(f2), by = ce_y(f2), bz = ce_z(f2);
                    T h = T(0);
                    sfor<bx + 1>([&](auto UX) {
                        sfor<by + 1>([&](auto UY) {
                            sfor<bz + 1>([&](auto UZ) {
                                constexpr int ux = TLNO_CI(UX), uy = TLNO_CI(UY), uz = TLNO_CI(UZ);
                                constexpr int fu = ce_flat(ce_x(f1) + ux, ce_y(f1) + uy, ce_z(f1) + uz) - OF;
                                h += hrr_coef<bx, ux>(X[0]) * hrr_coef<by, uy>(X[1]) * hrr_coef<bz, uz>(X[2]) *
                                     src(std::integral_constant<int, fu>{});
                            });
                        });
                    });
                    if constexpr (L2 <= 1) row += h;
                    else row += T(c_c2s.dense[L2][S2][c2]) * h;
                }
            });
            if constexpr (L1 <= 1) out += row;
            else out += T(c_c2s.dense[L1][S1][c1]) * row;
        }
    });
    return out;
}

struct QuartetGeom {
    double A[3], C[3];
    double AB[3], CD[3];
};

// Phase 1 + 2 for slice G (rows ia = G, G+TPQ, ...).
template <typename R, int LA, int LB, int LC, int LD, int G>
__device__ __forceinline__ void fast_slice(const PlanView& pv, int bra, int ket, bool active, const QuartetGeom& q,
                                           double fs_thr2, const float* rtab, R* __restrict__ ks) {
    using S = FastShape<LA, LB, LC, LD>;
    constexpr int ROWS = (S::NAS - G + S::TPQ - 1) / S::TPQ;
    R acc[ROWS > 0 ? ROWS : 1][S::NCS];
#pragma unroll
    for (int rr = 0; rr < ROWS; ++rr)
#pragma unroll
        for (int ic = 0; ic < S::NCS; ++ic) acc[rr][ic] = R(0);

    if (active) {
        const int npb = __ldg(pv.pair_nprim + bra), npk = __ldg(pv.pair_nprim + ket);
        const int ob = __ldg(pv.pair_prim_off + bra), ok = __ldg(pv.pair_prim_off + ket);
        // FP64: 48-byte records {p, Px, Py, Pz, w, 1/p} read as three 16-byte
        // vectors.  FP32: 24-byte records {p, P-A, w, 1/p} relative to the
        // pair's first centre, PQ = (P-A) - (Q-C) + (A-C).
        const double2* pb = reinterpret_cast<const double2*>(pv.prim + ob);
        const double2* pk = reinterpret_cast<const double2*>(pv.prim + ok);
        const float2* pb32 = reinterpret_cast<const float2*>(pv.prim32 + ob);
        const float2* pk32 = reinterpret_cast<const float2*>(pv.prim32 + ok);
        constexpr bool F32 = std::is_same<R, float>::value;
        const R ACx = R(q.A[0] - q.C[0]), ACy = R(q.A[1] - q.C[1]), ACz = R(q.A[2] - q.C[2]);
        // Primitive FASTSCHWARZ: a primitive quartet whose estimate product is
        // below the squared threshold contributes nothing (per lane; the
        // reference drops a SIMD packet only when every lane fails).
        const bool fs_on = fs_thr2 > 0.0;
        // Ket primitive outer, bra primitive inner: each lane gathers its own
        // ket record once per bra, and the bra records (the same for every
        // lane of the warp) are broadcast loads.
        for (int ik = 0; ik < npk; ++ik) {
            const double fsk = fs_on ? __ldg(pv.prim_fs + ok + ik) : 0.0;
            R qe, QCx, QCy, QCz, kw, kip;
            double kp_x = 0.0, kp_y = 0.0, kp_z = 0.0;
            if constexpr (F32) {
                const float2 u0 = __ldg(pk32 + 3 * ik), u1 = __ldg(pk32 + 3 * ik + 1), u2 = __ldg(pk32 + 3 * ik + 2);
                qe = u0.x; QCx = u0.y; QCy = u1.x; QCz = u1.y; kw = u2.x; kip = u2.y;
            } else {
                const double2 k0v = __ldg(pk + 3 * ik), k1v = __ldg(pk + 3 * ik + 1), k2v = __ldg(pk + 3 * ik + 2);
                kp_x = k0v.y; kp_y = k1v.x; kp_z = k1v.y;
                qe = R(k0v.x);
                QCx = R(kp_x - q.C[0]); QCy = R(kp_y - q.C[1]); QCz = R(kp_z - q.C[2]);
                kw = R(k2v.x); kip = R(k2v.y);
            }
            for (int ib = 0; ib < npb; ++ib) {
                if (fs_on && !(__ldg(pv.prim_fs + ob + ib) * fsk >= fs_thr2)) continue;
                R p, PAx, PAy, PAz, bw, bip, PQx, PQy, PQz;
                if constexpr (F32) {
                    const float2 u0 = __ldg(pb32 + 3 * ib), u1 = __ldg(pb32 + 3 * ib + 1), u2 = __ldg(pb32 + 3 * ib + 2);
                    p = u0.x; PAx = u0.y; PAy = u1.x; PAz = u1.y; bw = u2.x; bip = u2.y;
                    PQx = PAx - QCx + ACx; PQy = PAy - QCy + ACy; PQz = PAz - QCz + ACz;
                } else {
                    const double2 b0v = __ldg(pb + 3 * ib), b1v = __ldg(pb + 3 * ib + 1), b2v = __ldg(pb + 3 * ib + 2);
                    const double bp_x = b0v.y, bp_y = b1v.x, bp_z = b1v.y;
                    p = R(b0v.x);
                    PAx = R(bp_x - q.A[0]); PAy = R(bp_y - q.A[1]); PAz = R(bp_z - q.A[2]);
                    bw = R(b2v.x); bip = R(b2v.y);
                    PQx = R(bp_x - kp_x); PQy = R(bp_y - kp_y); PQz = R(bp_z - kp_z);
                }
                const R pqs = p + qe;
                // one reciprocal square root gives both 1/sqrt(p+q) and 1/(p+q)
                const R rs = rsqrt(pqs);
                const R inv = rs * rs;
                const R Targ = p * qe * inv * (PQx * PQx + PQy * PQy + PQz * PQz);
                R rt[S::N], wt[S::N];
                if constexpr (F32 && S::N <= 3) {
                    // FP32 interval polynomials staged in shared memory
                    rys_roots_smem32<S::N>(Targ, rtab, rt, wt);
                } else if constexpr (F32) {
                    // FP64 carve-out: roots and weights of N >= 4 (high-L)
                    // quartets come from the FP64 tables even in the FP32 pass
                    double rd[S::N], wd[S::N];
                    rys_roots_all<double, S::N>(double(Targ), rd, wd);
#pragma unroll
                    for (int r = 0; r < S::N; ++r) {
                        rt[r] = R(rd[r]);
                        wt[r] = R(wd[r]);
                    }
                } else {
                    rys_roots_all<R, S::N>(Targ, rt, wt);
                }
                const R pref = R(34.98683665524972497) * bw * kw * rs;
                const R qo = qe * inv, po = p * inv;
                const R hbp = R(0.5) * bip, hkp = R(0.5) * kip;
#pragma unroll
                for (int r = 0; r < S::N; ++r) {
                    const R t2 = rt[r];
                    const R b00 = R(0.5) * inv * t2;
                    const R b10 = hbp - hbp * qo * t2;
                    const R b01 = hkp - hkp * po * t2;
                    const R qt = qo * t2, pt = po * t2;
                    R g[3][S::GS];
                    const R c00[3] = {PAx - qt * PQx, PAy - qt * PQy, PAz - qt * PQz};
                    const R d00[3] = {QCx + pt * PQx, QCy + pt * PQy, QCz + pt * PQz};
#pragma unroll
                    for (int ax = 0; ax < 3; ++ax) {
                        R* G2 = g[ax];
                        G2[0] = (ax == 2) ? pref * wt[r] : R(1);
                        if (S::LAB > 0) G2[S::KS] = c00[ax] * G2[0];
#pragma unroll
                        for (int ii = 1; ii < S::LAB; ++ii)
                            G2[(ii + 1) * S::KS] = c00[ax] * G2[ii * S::KS] + R(ii) * b10 * G2[(ii - 1) * S::KS];
#pragma unroll
                        for (int k = 0; k < S::LCD; ++k) {
#pragma unroll
                            for (int ii = 0; ii <= S::LAB; ++ii) {
                                R v = d00[ax] * G2[ii * S::KS + k];
                                if (ii > 0) v += R(ii) * b00 * G2[(ii - 1) * S::KS + k];
                                if (k > 0) v += R(k) * b01 * G2[ii * S::KS + k - 1];
                                G2[ii * S::KS + k + 1] = v;
                            }
                        }
                    }
                    sfor<ROWS>([&](auto RR) {
                        constexpr int rr = TLNO_CI(RR);
                        constexpr int fa = S::OFA + G + rr * S::TPQ;
                        constexpr int xa = ce_x(fa), ya = ce_y(fa), za = ce_z(fa);
                        sfor<S::NCS>([&](auto IC) {
                            constexpr int ic = TLNO_CI(IC);
                            constexpr int fc = S::OFC + ic;
                            acc[rr][ic] += (g[0][xa * S::KS + ce_x(fc)] * g[1][ya * S::KS + ce_y(fc)]) *
                                           g[2][za * S::KS + ce_z(fc)];
                        });
                    });
                }
            }
        }
    }

    // Phase 2: ket transfer + projection of the owned rows (in R: the FP32
    // kernels keep the whole quartet in FP32 up to the FP64 atomics).
    const R CDr[3] = {R(q.CD[0]), R(q.CD[1]), R(q.CD[2])};
    sfor<ROWS>([&](auto RR) {
        constexpr int rr = TLNO_CI(RR);
        constexpr int ia = G + rr * S::TPQ;
        sfor<S::NSC>([&](auto SC) {
            sfor<S::NSD>([&](auto SD) {
                constexpr int sc = TLNO_CI(SC), sd = TLNO_CI(SD);
                ks[ia * S::NSCD + sc * S::NSD + sd] = pair_transfer<R, LC, LD, sc, sd, S::OFC>(
                    CDr, [&](auto FU) { return acc[rr][TLNO_CI(FU)]; });
            });
        });
    });
}

template <typename R, int LA, int LB, int LC, int LD, int G = 0>
__device__ __forceinline__ void fast_slice_dispatch(int g, const PlanView& pv, int bra, int ket, bool active,
                                                    const QuartetGeom& q, double fs_thr2, const float* rtab,
                                                    R* ks) {
    using S = FastShape<LA, LB, LC, LD>;
    if constexpr (G < S::TPQ) {
        if (g == G)
            fast_slice<R, LA, LB, LC, LD, G>(pv, bra, ket, active, q, fs_thr2, rtab, ks);
        else
            fast_slice_dispatch<R, LA, LB, LC, LD, G + 1>(g, pv, bra, ket, active, q, fs_thr2, rtab, ks);
    }
}

// Barrier and OR-vote over the TPQ warps of one group (named barrier
// 1 + group, so the groups of a CTA run independent control flow).
__device__ __forceinline__ void group_sync(int id, int nthreads) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}
__device__ __forceinline__ bool group_any(bool pred, int id, int nthreads) {
    int r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\tsetp.ne.s32 p, %1, 0;\n\tbar.red.or.pred q, %2, %3, p;\n\tselp.s32 %0, 1, 0, q;\n\t}"
        : "=r"(r)
        : "r"(pred ? 1 : 0), "r"(id), "r"(nthreads)
        : "memory");
    return r != 0;
}

// The lightest classes (at most 9 radial accumulators per thread) are
// latency-bound on their gathers: a register cap of 4 resident CTAs per SM
// (FP64) or 6 (FP32) buys more warps than it costs (measured on 200 waters);
// classes with larger accumulator blocks would spill under it.  FP32 (ps|ss)
// takes 7 (cfg4: 1199 -> 1119 ms; 7 or 8 is slower or equal on the other
// light classes).
template <typename R, int LA, int LB, int LC, int LD>
__host__ __device__ constexpr int fast_min_blocks() {
    using S = FastShape<LA, LB, LC, LD>;
    // unsliced FP32 classes with larger accumulator blocks: 3 resident CTAs
    // instead of the 2 their ~200 registers allow, 4 for (pp|ps), (ds|ps),
    // (dp|ss), (ds|ds), (dd|ss) (measured per class on 200 waters; 4 is
    // slower on the others)
    if (S::TPQ == 1 && S::NAS * S::NCS > 9) {
        if (!std::is_same<R, float>::value) return 1;
        constexpr bool four = (LA == 1 && LB == 1 && LC == 1 && LD == 0) || (LA == 2 && LB == 0 && LC == 1 && LD == 0) ||
                              (LA == 2 && LB == 1 && LC == 0 && LD == 0) || (LA == 2 && LB == 0 && LC == 2 && LD == 0) ||
                              (LA == 2 && LB == 2 && LC == 0 && LD == 0);
        return four ? 4 : 3;
    }
    if (!(S::TPQ == 1 && S::NAS * S::NCS <= 9)) return 1;
    if (!std::is_same<R, float>::value) return 4;
    return (LA == 1 && LB == 0 && LC == 0 && LD == 0) ? 7 : 6;
}

// Where a bra-group class keeps the per-tile density values of a lane:
// 0 none (no bra groups), 1 registers, 2 shared memory.  Shared memory where
// registers are tight (FP64, and the capped FP32 classes: 3-10% faster on the
// s/p classes of 400 waters); registers for the uncapped FP32 classes, where
// the extra shared memory costs resident CTAs (+18% on (pp|ps)).
template <typename R, int LA, int LB, int LC, int LD>
__host__ __device__ constexpr int fast_pre_mode() {
    using S = FastShape<LA, LB, LC, LD>;
    if (S::PRE_VALS == 0) return 0;
    if (std::is_same<R, double>::value) return 2;
    return fast_min_blocks<R, LA, LB, LC, LD>() > 1 ? 2 : 1;
}

template <typename R, int LA, int LB, int LC, int LD>
__global__ void __launch_bounds__(32 * FastShape<LA, LB, LC, LD>::WARPS, fast_min_blocks<R, LA, LB, LC, LD>())
    eri_fast_jk_kernel(PlanView pv, ClassLaunch cl) {
    using S = FastShape<LA, LB, LC, LD>;
    extern __shared__ double fast_smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int grp = warp / S::TPQ, g = warp % S::TPQ;
    // A quartet owned by one thread keeps its (a0|cd) rows in registers; a
    // sliced quartet exchanges them through shared memory.
    R ks_reg[S::TPQ == 1 ? S::NAS * S::NSCD : 1];
    R* ks;
    if constexpr (S::TPQ == 1)
        ks = ks_reg;
    else
        ks = reinterpret_cast<R*>(fast_smem) + (grp * 32 + lane) * S::LANE_STRIDE;
    const double thr = (cl.prec_mode != 0) ? cl.tau_mix / fmax(*cl.dmax, 1e-300) : 0.0;
    const int bar_id = 1 + grp, bar_n = 32 * S::TPQ;
    // FP32 kernels with N <= 3 stage their Rys interval polynomials in shared
    // memory behind the row-exchange buffer.
    const float* rtab = nullptr;
    int smem_used = S::SMEM_DOUBLES * 8;  // bytes
    if constexpr (std::is_same<R, float>::value && S::N <= 3) {
        float* t = reinterpret_cast<float*>(fast_smem + S::SMEM_DOUBLES);
        const int n4 = c_tabs.rys32_nint[S::N] * (kRys32CoefDev * 2 * S::N) / 4;
        const float4* src = reinterpret_cast<const float4*>(c_tabs.rys32[S::N]);
        for (int i = threadIdx.x; i < n4; i += blockDim.x) reinterpret_cast<float4*>(t)[i] = __ldg(src + i);
        __syncthreads();
        rtab = t;
        smem_used += n4 * 16;
    }
    // this warp's slots of the per-tile density values (shared-memory mode)
    constexpr int PRE_MODE = fast_pre_mode<R, LA, LB, LC, LD>();
    R* pre = reinterpret_cast<R*>(reinterpret_cast<unsigned char*>(fast_smem) + smem_used) +
             (PRE_MODE == 2 ? warp * 32 * S::PRE_VALS : 0);
    __shared__ int s_chunk[S::BBQ];
    const int ntiles = cl.tile_end - cl.tile_begin;
    double csum = 0.0;  // ERI checksum stream: this thread's share

    // tiles per fetch (per-class tuning; 0 = the default)
    const int chunk = cl.chunk > 0 ? cl.chunk : kTileChunk;
    // Dynamic schedule: every warp group takes `chunk` consecutive tiles
    // (one bra pair x 32 kets each) from the launch counter, so all groups
    // work inside one moving window of the schedule and the density, J and
    // K rows of the bras in flight stay in L2.  The first tile's block comes
    // from a binary search, the next ones from walking the prefix forward.
    for (;;) {
        int c0;
        if constexpr (S::TPQ == 1) {
            c0 = (lane == 0) ? atomicAdd(cl.counter, chunk) : 0;
            c0 = __shfl_sync(0xffffffffu, c0, 0);
        } else {
            if (g == 0 && lane == 0) s_chunk[grp] = atomicAdd(cl.counter, chunk);
            group_sync(bar_id, bar_n);
            c0 = s_chunk[grp];
            group_sync(bar_id, bar_n);
        }
        if (c0 >= ntiles) break;
        const int c1 = min(c0 + chunk, ntiles);
        int b = find_block(cl.tile_prefix, cl.n_blocks, cl.tile_begin + c0);
        int next = __ldg(cl.tile_prefix + b + 1);
    for (int tile = cl.tile_begin + c0; tile < cl.tile_begin + c1; ++tile) {
        while (tile >= next) {
            ++b;
            next = __ldg(cl.tile_prefix + b + 1);
        }
        const int kb = tile - __ldg(cl.tile_prefix + b);
        const BlockDesc bd = cl.blocks[b];
        const int j = kb * 32 + lane;
        const bool lane_ok = j < bd.nket;
        const int ket = bd.ket0 + (lane_ok ? j : 0);

        // Quick test on the Schwarz products alone: a tile without any quartet
        // for this launch (bound, triangle, precision pass) is left before
        // the ket geometry is loaded.
        const double qket = __ldg(pv.pair_Q + ket);
        const int mol = pv.pair_mol ? __ldg(pv.pair_mol + ket) : 0;
        // the density screen raises the Schwarz cutoff of this build
        const double tau_t = cl.den.mode ? density_tau_min(cl, mol) : cl.tau;
        {
            bool act = false;
            for (int ib = 0; ib < S::GB && ib < bd.nbra; ++ib) {
                const int bra = __ldg(cl.bra_list + bd.bra0 + ib);
                if (!lane_ok || (cl.same && bd.koff + j > bra - bd.xbeg)) continue;
                const double qq = __ldg(pv.pair_Q + bra) * qket;
                bool a = qq >= tau_t;
                if (cl.prec_mode == 1) a = a && qq >= thr;
                if (cl.prec_mode == 2) a = a && !(qq >= thr);
                act = act || a;
            }
            bool any_tile;
            if constexpr (S::TPQ > 1)
                any_tile = group_any(act, bar_id, bar_n);
            else
                any_tile = __any_sync(0xffffffffu, act);
            if (!any_tile) continue;
        }

        // ket side, once per tile
        const int C = __ldg(pv.pair_A + ket), D = __ldg(pv.pair_B + ket);
        QuartetGeom q;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            q.C[k] = __ldg(pv.shell_xyz + 3 * C + k);
            q.CD[k] = q.C[k] - __ldg(pv.shell_xyz + 3 * D + k);
        }
        const int M = pv.mol_M ? __ldg(pv.mol_M + mol) : cl.M;
        const long long mbase = pv.mol_mat_off ? __ldg(pv.mol_mat_off + mol) : 0;
        const double* Dm = cl.dens + mbase;
        double* Jm = cl.J + mbase;
        double* Km = cl.K + mbase;
        // FP32 kernels gather from the FP32 copy of the density
        const float* Dm32 = cl.dens32 + mbase;
        auto dm = [&](int r, int c) {
            if constexpr (std::is_same<R, float>::value)
                return R(__ldg(Dm32 + (long long)r * M + c));
            else
                return __ldg(Dm + (long long)r * M + c);
        };
        const int c0 = __ldg(pv.shell_sph + C), d0 = __ldg(pv.shell_sph + D);

        // Sums carried across the bras of a block (they share the first
        // shell A): J[cd], K[ac], K[ad] of this lane's ket.
        constexpr bool CARRY = S::GB > 1;
        R jcd[CARRY ? S::NSCD : 1];
        R kacc[CARRY ? S::NSA : 1][CARRY ? S::NSC : 1];
        R kadc[CARRY ? S::NSA : 1][CARRY ? S::NSD : 1];
        if constexpr (CARRY) {
#pragma unroll
            for (int t = 0; t < S::NSCD; ++t) jcd[t] = 0.0;
#pragma unroll
            for (int a = 0; a < S::NSA; ++a) {
#pragma unroll
                for (int c = 0; c < S::NSC; ++c) kacc[a][c] = 0.0;
#pragma unroll
                for (int d = 0; d < S::NSD; ++d) kadc[a][d] = 0.0;
            }
        }
        // The bras of a block share shell A, so the lane's D[a, c], D[a, d]
        // and D[c, d] are the same for every bra of it: they are gathered once
        // per tile, into registers or this lane's shared-memory slots
        // [k * 32 + lane].
        constexpr bool PRE = PRE_MODE != 0;
        R preg[PRE_MODE == 1 ? S::PRE_VALS : 1];
        auto pre_at = [&](int k) -> R& {
            if constexpr (PRE_MODE == 1) return preg[k];
            else return pre[k * 32 + lane];
        };
        if constexpr (PRE) {
            const int a0b = __ldg(pv.shell_sph + __ldg(pv.pair_A + __ldg(cl.bra_list + bd.bra0)));
            if (cl.want_k) {
#pragma unroll
                for (int sa = 0; sa < S::NSA; ++sa) {
#pragma unroll
                    for (int sc = 0; sc < S::NSC; ++sc) pre_at(sa * S::NSC + sc) = dm(a0b + sa, c0 + sc);
#pragma unroll
                    for (int sd = 0; sd < S::NSD; ++sd)
                        pre_at(S::NSA * S::NSC + sa * S::NSD + sd) = dm(a0b + sa, d0 + sd);
                }
            }
            if (cl.want_j) {
#pragma unroll
                for (int t = 0; t < S::NSCD; ++t)
                    pre_at(S::NSA * (S::NSC + S::NSD) + t) = dm(c0 + t / S::NSD, d0 + t % S::NSD);
            }
        }
        bool touched = false;
        int a0 = 0;

        for (int ib = 0; ib < S::GB && ib < bd.nbra; ++ib) {
            const int bra = __ldg(cl.bra_list + bd.bra0 + ib);
            const int i = bra - bd.xbeg;
            const int A = __ldg(pv.pair_A + bra), B = __ldg(pv.pair_B + bra);
            bool active = lane_ok && !(cl.same && bd.koff + j > i);
            // density screen: Coulomb and exchange contributions kept apart
            R jon = R(1), kon = R(1);
            if (active) {
                const double qq = __ldg(pv.pair_Q + bra) * qket;
                active = qq >= cl.tau;
                if (cl.prec_mode == 1) active = active && qq >= thr;
                if (cl.prec_mode == 2) active = active && !(qq >= thr);
                if (active && cl.den.mode) {
                    bool lj, lk;
                    density_live(cl, pv, mol, A, B, C, D, qq, lj, lk);
                    active = lj || lk;
                    jon = lj ? R(1) : R(0);
                    kon = lk ? R(1) : R(0);
                }
            }
            bool any;
            if constexpr (S::TPQ > 1)
                any = group_any(active, bar_id, bar_n);
            else
                any = __any_sync(0xffffffffu, active);
            if (!any) continue;
            touched = touched || active;

#pragma unroll
            for (int k = 0; k < 3; ++k) {
                q.A[k] = __ldg(pv.shell_xyz + 3 * A + k);
                q.AB[k] = q.A[k] - __ldg(pv.shell_xyz + 3 * B + k);
            }
            fast_slice_dispatch<R, LA, LB, LC, LD>(g, pv, bra, ket, active, q, cl.fs_thr2, rtab, ks);
            if constexpr (S::TPQ > 1) group_sync(bar_id, bar_n);

            // ---- bra transfer + projection per owned ket column, digestion ----
            a0 = __ldg(pv.shell_sph + A);
            const int b0 = __ldg(pv.shell_sph + B);
            R f = active ? R(1) : R(0);
            if (A == B) f *= R(0.5);
            if (C == D) f *= R(0.5);
            if (bra == ket) f *= R(0.5);
            const R fj = R(4) * f * jon, fk = R(2) * f * kon;
            const R ABr[3] = {R(q.AB[0]), R(q.AB[1]), R(q.AB[2])};

            R jab[S::NSAB];
#pragma unroll
            for (int e = 0; e < S::NSAB; ++e) jab[e] = R(0);
            if (active) {
                R kad[CARRY ? 1 : S::NSA][CARRY ? 1 : S::NSD];
                R kbd[S::NSB][S::NSD];
                if constexpr (!CARRY) {
#pragma unroll
                    for (int a = 0; a < S::NSA; ++a)
#pragma unroll
                        for (int d = 0; d < S::NSD; ++d) kad[a][d] = 0.0;
                }
#pragma unroll
                for (int bq = 0; bq < S::NSB; ++bq)
#pragma unroll
                    for (int d = 0; d < S::NSD; ++d) kbd[bq][d] = 0.0;
                sfor<S::NSC>([&](auto SC) {
                    constexpr int sc = TLNO_CI(SC);
                    R kac[CARRY ? 1 : S::NSA], kbc[S::NSB];
                    if constexpr (!CARRY) {
#pragma unroll
                        for (int a = 0; a < S::NSA; ++a) kac[a] = 0.0;
                    }
#pragma unroll
                    for (int bq = 0; bq < S::NSB; ++bq) kbc[bq] = 0.0;
                    bool own_sc = false;
                    sfor<S::NSD>([&](auto SD) {
                        constexpr int sd = TLNO_CI(SD);
                        constexpr int t = sc * S::NSD + sd;
                        const bool own = S::BY_SC ? (sc % S::TPQ == g) : (t % S::TPQ == g);
                        if (!own) return;
                        own_sc = true;
                        R V[S::NSAB];
                        sfor<S::NSA>([&](auto SA) {
                            sfor<S::NSB>([&](auto SB) {
                                constexpr int sa = TLNO_CI(SA), sb = TLNO_CI(SB);
                                V[sa * S::NSB + sb] = pair_transfer<R, LA, LB, sa, sb, S::OFA>(
                                    ABr, [&](auto FU) { return ks[TLNO_CI(FU) * S::NSCD + t]; });
                            });
                        });
                        if (cl.checksum) {
#pragma unroll
                            for (int e = 0; e < S::NSAB; ++e)
                                if (canonical_element(A == B, C == D, bra == ket, a0, e / S::NSB, b0, e % S::NSB, c0,
                                                      sc, d0, sd))
                                    csum += double(V[e]);
                        }
                        if (cl.want_j) {
                            R s = R(0);
#pragma unroll
                            for (int e = 0; e < S::NSAB; ++e) s += V[e] * R(dm(a0 + e / S::NSB, b0 + e % S::NSB));
                            if constexpr (CARRY)
                                jcd[t] += fj * s;
                            else
                                atomicAdd(Jm + (long long)(c0 + sc) * M + d0 + sd, double(fj * s));
                            R dcd;
                            if constexpr (PRE) dcd = pre_at(S::NSA * (S::NSC + S::NSD) + t);
                            else dcd = R(dm(c0 + sc, d0 + sd));
#pragma unroll
                            for (int e = 0; e < S::NSAB; ++e) jab[e] += V[e] * dcd;
                        }
                        if (cl.want_k) {
                            // D[b, d] and D[b, c] of this column, gathered once
                            R dbd[S::NSB], dbc[S::NSB];
#pragma unroll
                            for (int sb = 0; sb < S::NSB; ++sb) {
                                dbd[sb] = R(dm(b0 + sb, d0 + sd));
                                dbc[sb] = R(dm(b0 + sb, c0 + sc));
                            }
#pragma unroll
                            for (int sa = 0; sa < S::NSA; ++sa) {
                                R dad, dac;
                                if constexpr (PRE) {
                                    dad = pre_at(S::NSA * S::NSC + sa * S::NSD + sd);
                                    dac = pre_at(sa * S::NSC + sc);
                                } else {
                                    dad = R(dm(a0 + sa, d0 + sd));
                                    dac = R(dm(a0 + sa, c0 + sc));
                                }
                                R sac = R(0), sad = R(0);
#pragma unroll
                                for (int sb = 0; sb < S::NSB; ++sb) {
                                    const R v = V[sa * S::NSB + sb];
                                    sac += v * dbd[sb];
                                    sad += v * dbc[sb];
                                    kbc[sb] += v * dad;
                                    kbd[sb][sd] += v * dac;
                                }
                                if constexpr (CARRY) {
                                    kacc[sa][sc] += fk * sac;
                                    kadc[sa][sd] += fk * sad;
                                } else {
                                    kac[sa] += sac;
                                    kad[sa][sd] += sad;
                                }
                            }
                        }
                    });
                    if (cl.want_k && own_sc) {
                        if constexpr (!CARRY) {
#pragma unroll
                            for (int sa = 0; sa < S::NSA; ++sa)
                                atomicAdd(Km + (long long)(a0 + sa) * M + c0 + sc, double(fk * kac[sa]));
                        }
#pragma unroll
                        for (int sb = 0; sb < S::NSB; ++sb)
                            atomicAdd(Km + (long long)(b0 + sb) * M + c0 + sc, double(fk * kbc[sb]));
                    }
                });
                if (cl.want_k) {
                    sfor<S::NSD>([&](auto SD) {
                        constexpr int sd = TLNO_CI(SD);
                        bool own_d = false;
#pragma unroll
                        for (int sc = 0; sc < S::NSC; ++sc)
                            own_d = own_d || (S::BY_SC ? (sc % S::TPQ == g) : ((sc * S::NSD + sd) % S::TPQ == g));
                        if (!own_d) return;
                        if constexpr (!CARRY) {
#pragma unroll
                            for (int sa = 0; sa < S::NSA; ++sa)
                                atomicAdd(Km + (long long)(a0 + sa) * M + d0 + sd, double(fk * kad[sa][sd]));
                        }
#pragma unroll
                        for (int sb = 0; sb < S::NSB; ++sb)
                            atomicAdd(Km + (long long)(b0 + sb) * M + d0 + sd, double(fk * kbd[sb][sd]));
                    });
                }
            }
            if (cl.want_j) {
                // J[ab]: every lane of the warp shares the bra pair.
#pragma unroll
                for (int e = 0; e < S::NSAB; ++e) {
                    R s = fj * jab[e];
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
                    if (lane == 0 && s != R(0)) atomicAdd(Jm + (long long)(a0 + e / S::NSB) * M + b0 + e % S::NSB, double(s));
                }
            }
            if constexpr (S::TPQ > 1) group_sync(bar_id, bar_n);
        }

        if constexpr (CARRY) {
            // Flush the block's carried ket-side sums (a0 is common to the block).
            if (touched) {
                if (cl.want_j) {
#pragma unroll
                    for (int t = 0; t < S::NSCD; ++t)
                        atomicAdd(Jm + (long long)(c0 + t / S::NSD) * M + d0 + t % S::NSD, double(jcd[t]));
                }
                if (cl.want_k) {
#pragma unroll
                    for (int sa = 0; sa < S::NSA; ++sa) {
#pragma unroll
                        for (int sc = 0; sc < S::NSC; ++sc) atomicAdd(Km + (long long)(a0 + sa) * M + c0 + sc, double(kacc[sa][sc]));
#pragma unroll
                        for (int sd = 0; sd < S::NSD; ++sd) atomicAdd(Km + (long long)(a0 + sa) * M + d0 + sd, double(kadc[sa][sd]));
                    }
                }
            }
        }
    }
    }
    if (cl.checksum) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) csum += __shfl_xor_sync(0xffffffffu, csum, o);
        if (lane == 0 && csum != 0.0) atomicAdd(cl.checksum, csum);
    }
}

// Launch geometry of class (la lb|lc ld) for the host.
template <int LA, int LB, int LC, int LD>
constexpr int fast_warps() { return FastShape<LA, LB, LC, LD>::WARPS; }
template <int LA, int LB, int LC, int LD>
constexpr int fast_bras() { return FastShape<LA, LB, LC, LD>::GB; }
template <int LA, int LB, int LC, int LD>
constexpr int fast_smem_bytes() { return FastShape<LA, LB, LC, LD>::SMEM_DOUBLES * 8; }
template <int LA, int LB, int LC, int LD>
constexpr int fast_roots() { return FastShape<LA, LB, LC, LD>::N; }
template <int LA, int LB, int LC, int LD>
constexpr int fast_pre_bytes(bool fp32) {
    using S = FastShape<LA, LB, LC, LD>;
    return fp32 ? (fast_pre_mode<float, LA, LB, LC, LD>() == 2 ? S::WARPS * 32 * S::PRE_VALS * 4 : 0)
                : (fast_pre_mode<double, LA, LB, LC, LD>() == 2 ? S::WARPS * 32 * S::PRE_VALS * 8 : 0);
}

}  // namespace dev
}  // namespace tlno_gpu
