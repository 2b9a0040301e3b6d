// Thread-per-quartet Rys ERI + J/K kernel for the light angular-momentum
// classes, with the class fixed at compile time so the 2-D recurrences, the
// contracted radial accumulators, the horizontal transfer and the spherical
// projection all live in registers.
//
// Tile: one warp per bra shell pair, 32 consecutive ket shell pairs (one per
// lane), `bb` warps per CTA on consecutive bra pairs; kets are sorted by
// Schwarz bound so a lane whose quartet fails the bound ends the warp's row.
// J[ab] is reduced over the warp before its atomic update; the other five
// digestion targets are updated per lane with FP64 atomics.
#pragma once

#include "eri_common.cuh"

namespace tlno_gpu {
namespace dev {

__host__ __device__ constexpr int ce_ncart(int L) { return (L + 1) * (L + 2) / 2; }
__host__ __device__ constexpr int ce_nsph(int L) { return 2 * L + 1; }
__host__ __device__ constexpr int ce_off(int L) { return L * (L + 1) * (L + 2) / 6; }
__host__ __device__ constexpr int ce_cum(int L) { return (L + 1) * (L + 2) * (L + 3) / 6; }
// Cartesian exponents of flat index f (reference order).
__host__ __device__ constexpr int ce_L(int f) {
    int L = 0;
    while (ce_cum(L) <= f) ++L;
    return L;
}
__host__ __device__ constexpr int ce_x(int f) {
    const int L = ce_L(f);
    int loc = f - ce_off(L);
    int x = L;
    while (loc >= L - x + 1) { loc -= L - x + 1; --x; }
    return x;
}
__host__ __device__ constexpr int ce_y(int f) {
    const int L = ce_L(f);
    int loc = f - ce_off(L);
    int x = L;
    while (loc >= L - x + 1) { loc -= L - x + 1; --x; }
    return L - x - loc;
}
__host__ __device__ constexpr int ce_z(int f) { return ce_L(f) - ce_x(f) - ce_y(f); }
__host__ __device__ constexpr int ce_flat(int x, int y, int z) {
    return ce_off(x + y + z) + (y + z) * (y + z + 1) / 2 + z;
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
};

// C(b,u) * x^(b-u) for small b, u (compile-time b, u).
template <typename T>
__device__ __forceinline__ T hrr_coef(int b, int u, T x) {
    T c = T(1);
    // binomial
    int num = 1, den = 1;
    for (int i = 0; i < u; ++i) { num *= (b - i); den *= (i + 1); }
    c = T(num / den);
    for (int i = 0; i < b - u; ++i) c *= x;
    return c;
}

template <typename R, int LA, int LB, int LC, int LD>
__global__ void __launch_bounds__(128) eri_fast_jk_kernel(PlanView pv, ClassLaunch cl) {
    using S = FastShape<LA, LB, LC, LD>;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const double thr = (cl.prec_mode != 0) ? cl.tau_mix / fmax(*cl.dmax, 1e-300) : 0.0;
    for (int tile = cl.tile_begin + blockIdx.x; tile < cl.tile_end; tile += gridDim.x) {
        const int b = find_block(cl.tile_prefix, cl.n_blocks, tile);
        const int kb = tile - __ldg(cl.tile_prefix + b);
        const BlockDesc bd = cl.blocks[b];
        if (warp >= bd.nbra) continue;
        const int i = bd.ilocal0 + warp;
        const int j = kb * 32 + lane;
        const int bra = bd.bra0 + warp;
        const double qi = pv.pair_Q[bra];
        bool active = j < bd.nket && !(cl.same && j > i);
        const int ket = bd.ket0 + (active ? j : 0);
        if (active) {
            const double qq = qi * pv.pair_Q[ket];
            active = qq >= cl.tau;
            if (cl.prec_mode == 1) active = active && qq >= thr;
            if (cl.prec_mode == 2) active = active && !(qq >= thr);
        }
        if (!__any_sync(0xffffffffu, active)) continue;

        const int A = pv.pair_A[bra], B = pv.pair_B[bra];
        const int C = pv.pair_A[ket], D = pv.pair_B[ket];
        const double Ax = pv.shell_xyz[3 * A], Ay = pv.shell_xyz[3 * A + 1], Az = pv.shell_xyz[3 * A + 2];
        const double Cx = pv.shell_xyz[3 * C], Cy = pv.shell_xyz[3 * C + 1], Cz = pv.shell_xyz[3 * C + 2];

        R Tr[S::NAS * S::NCS];
#pragma unroll
        for (int e = 0; e < S::NAS * S::NCS; ++e) Tr[e] = R(0);

        if (active) {
            const int npb = pv.pair_nprim[bra], npk = pv.pair_nprim[ket];
            const DPrimPair* pb = pv.prim + pv.pair_prim_off[bra];
            const DPrimPair* pk = pv.prim + pv.pair_prim_off[ket];
            for (int ib = 0; ib < npb; ++ib) {
                const DPrimPair bp = pb[ib];
                const R p = R(bp.p);
                const R PAx = R(bp.Px - Ax), PAy = R(bp.Py - Ay), PAz = R(bp.Pz - Az);
                for (int ik = 0; ik < npk; ++ik) {
                    const DPrimPair kp = pk[ik];
                    const R q = R(kp.p);
                    const R pqs = p + q;
                    const R inv = R(1) / pqs;
                    const R PQx = R(bp.Px - kp.Px), PQy = R(bp.Py - kp.Py), PQz = R(bp.Pz - kp.Pz);
                    const R Targ = p * q * inv * (PQx * PQx + PQy * PQy + PQz * PQz);
                    R rt[S::N], wt[S::N];
                    rys_roots_all<R, S::N>(Targ, rt, wt);
                    const R pref = R(34.98683665524972497) * R(bp.w) * R(kp.w) / sqrt(pqs);
                    const R qo = q * inv, po = p * inv;
                    const R QCx = R(kp.Px - Cx), QCy = R(kp.Py - Cy), QCz = R(kp.Pz - Cz);
#pragma unroll
                    for (int r = 0; r < S::N; ++r) {
                        const R t2 = rt[r];
                        const R b00 = R(0.5) * inv * t2;
                        const R b10 = R(0.5) * R(bp.invp) * (R(1) - qo * t2);
                        const R b01 = R(0.5) * R(kp.invp) * (R(1) - po * t2);
                        R G[3][S::GS];
                        const R c00[3] = {PAx - qo * PQx * t2, PAy - qo * PQy * t2, PAz - qo * PQz * t2};
                        const R d00[3] = {QCx + po * PQx * t2, QCy + po * PQy * t2, QCz + po * PQz * t2};
#pragma unroll
                        for (int ax = 0; ax < 3; ++ax) {
                            R* g = G[ax];
                            g[0] = (ax == 2) ? pref * wt[r] : R(1);
                            if (S::LAB > 0) g[S::KS] = c00[ax] * g[0];
#pragma unroll
                            for (int ii = 1; ii < S::LAB; ++ii)
                                g[(ii + 1) * S::KS] = c00[ax] * g[ii * S::KS] + R(ii) * b10 * g[(ii - 1) * S::KS];
#pragma unroll
                            for (int k = 0; k < S::LCD; ++k) {
#pragma unroll
                                for (int ii = 0; ii <= S::LAB; ++ii) {
                                    R v = d00[ax] * g[ii * S::KS + k];
                                    if (ii > 0) v += R(ii) * b00 * g[(ii - 1) * S::KS + k];
                                    if (k > 0) v += R(k) * b01 * g[ii * S::KS + k - 1];
                                    g[ii * S::KS + k + 1] = v;
                                }
                            }
                        }
#pragma unroll
                        for (int ia = 0; ia < S::NAS; ++ia) {
#pragma unroll
                            for (int ic = 0; ic < S::NCS; ++ic) {
                                const int fa = S::OFA + ia, fc = S::OFC + ic;
                                Tr[ia * S::NCS + ic] += G[0][ce_x(fa) * S::KS + ce_x(fc)] *
                                                        G[1][ce_y(fa) * S::KS + ce_y(fc)] *
                                                        G[2][ce_z(fa) * S::KS + ce_z(fc)];
                            }
                        }
                    }
                }
            }
        }

        // Ket transfer K[ia][c][d] = sum_u C(d,u) CD^(d-u) T[ia][c+u], then the
        // ket spherical projection, then the bra transfer and projection.
        const double* xd = pv.shell_xyz + 3 * D;
        const double* xb = pv.shell_xyz + 3 * B;
        const double CD[3] = {Cx - xd[0], Cy - xd[1], Cz - xd[2]};
        const double AB[3] = {Ax - xb[0], Ay - xb[1], Az - xb[2]};
        constexpr int NSAB = S::NSA * S::NSB, NSCD = S::NSC * S::NSD;
        double Ks[S::NAS * NSCD];
#pragma unroll
        for (int ia = 0; ia < S::NAS; ++ia) {
            double Kc[S::NCC * S::NCD];
#pragma unroll
            for (int c = 0; c < S::NCC; ++c)
#pragma unroll
                for (int d = 0; d < S::NCD; ++d) {
                    const int fc = ce_off(LC) + c, fd = ce_off(LD) + d;
                    const int cxp = ce_x(fc), cyp = ce_y(fc), czp = ce_z(fc);
                    const int dx = ce_x(fd), dy = ce_y(fd), dz = ce_z(fd);
                    double s = 0.0;
#pragma unroll
                    for (int ux = 0; ux <= dx; ++ux)
#pragma unroll
                        for (int uy = 0; uy <= dy; ++uy)
#pragma unroll
                            for (int uz = 0; uz <= dz; ++uz) {
                                const int fcu = ce_flat(cxp + ux, cyp + uy, czp + uz) - S::OFC;
                                s += hrr_coef<double>(dx, ux, CD[0]) * hrr_coef<double>(dy, uy, CD[1]) *
                                     hrr_coef<double>(dz, uz, CD[2]) * double(Tr[ia * S::NCS + fcu]);
                            }
                    Kc[c * S::NCD + d] = s;
                }
#pragma unroll
            for (int sc = 0; sc < S::NSC; ++sc)
#pragma unroll
                for (int sd = 0; sd < S::NSD; ++sd) {
                    double s = 0.0;
#pragma unroll
                    for (int c = 0; c < S::NCC; ++c)
#pragma unroll
                        for (int d = 0; d < S::NCD; ++d) {
                            if ((LC <= 1 && c != sc) || (LD <= 1 && d != sd)) continue;
                            const double kc = (LC <= 1) ? 1.0 : c_c2s.dense[LC][sc][c];
                            const double kd = (LD <= 1) ? 1.0 : c_c2s.dense[LD][sd][d];
                            s += kc * kd * Kc[c * S::NCD + d];
                        }
                    Ks[ia * NSCD + sc * S::NSD + sd] = s;
                }
        }
        double V[NSAB * NSCD];
#pragma unroll
        for (int t = 0; t < NSCD; ++t) {
            double Vc[S::NCA * S::NCB];
#pragma unroll
            for (int a = 0; a < S::NCA; ++a)
#pragma unroll
                for (int bq = 0; bq < S::NCB; ++bq) {
                    const int fa = ce_off(LA) + a, fb = ce_off(LB) + bq;
                    const int axp = ce_x(fa), ayp = ce_y(fa), azp = ce_z(fa);
                    const int bx = ce_x(fb), by = ce_y(fb), bz = ce_z(fb);
                    double s = 0.0;
#pragma unroll
                    for (int ux = 0; ux <= bx; ++ux)
#pragma unroll
                        for (int uy = 0; uy <= by; ++uy)
#pragma unroll
                            for (int uz = 0; uz <= bz; ++uz) {
                                const int fau = ce_flat(axp + ux, ayp + uy, azp + uz) - S::OFA;
                                s += hrr_coef<double>(bx, ux, AB[0]) * hrr_coef<double>(by, uy, AB[1]) *
                                     hrr_coef<double>(bz, uz, AB[2]) * Ks[fau * NSCD + t];
                            }
                    Vc[a * S::NCB + bq] = s;
                }
#pragma unroll
            for (int sa = 0; sa < S::NSA; ++sa)
#pragma unroll
                for (int sb = 0; sb < S::NSB; ++sb) {
                    double s = 0.0;
#pragma unroll
                    for (int a = 0; a < S::NCA; ++a)
#pragma unroll
                        for (int bq = 0; bq < S::NCB; ++bq) {
                            if ((LA <= 1 && a != sa) || (LB <= 1 && bq != sb)) continue;
                            const double ka = (LA <= 1) ? 1.0 : c_c2s.dense[LA][sa][a];
                            const double kb = (LB <= 1) ? 1.0 : c_c2s.dense[LB][sb][bq];
                            s += ka * kb * Vc[a * S::NCB + bq];
                        }
                    V[(sa * S::NSB + sb) * NSCD + t] = s;
                }
        }

        // ---- digestion ----
        const int mol = pv.pair_mol ? pv.pair_mol[bra] : 0;
        const int M = pv.mol_M ? pv.mol_M[mol] : cl.M;
        const long long mbase = pv.mol_mat_off ? pv.mol_mat_off[mol] : 0;
        const double* Dm = cl.dens + mbase;
        double* Jm = cl.J + mbase;
        double* Km = cl.K + mbase;
        const int a0 = pv.shell_sph[A], b0 = pv.shell_sph[B];
        const int c0 = pv.shell_sph[C], d0 = pv.shell_sph[D];
        double f = active ? 1.0 : 0.0;
        if (A == B) f *= 0.5;
        if (C == D) f *= 0.5;
        if (bra == ket) f *= 0.5;
        if (cl.want_j) {
            double Pab[NSAB];
#pragma unroll
            for (int e = 0; e < NSAB; ++e) Pab[e] = __ldg(Dm + (long long)(a0 + e / S::NSB) * M + b0 + e % S::NSB);
#pragma unroll
            for (int sab = 0; sab < NSAB; ++sab) {
                double s = 0.0;
                if (active) {
#pragma unroll
                    for (int t = 0; t < NSCD; ++t)
                        s += V[sab * NSCD + t] * __ldg(Dm + (long long)(c0 + t / S::NSD) * M + d0 + t % S::NSD);
                }
                s *= 4.0 * f;
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
                if (lane == 0) atomicAdd(Jm + (long long)(a0 + sab / S::NSB) * M + b0 + sab % S::NSB, s);
            }
            if (active) {
#pragma unroll
                for (int t = 0; t < NSCD; ++t) {
                    double s = 0.0;
#pragma unroll
                    for (int sab = 0; sab < NSAB; ++sab) s += V[sab * NSCD + t] * Pab[sab];
                    atomicAdd(Jm + (long long)(c0 + t / S::NSD) * M + d0 + t % S::NSD, 4.0 * f * s);
                }
            }
        }
        if (cl.want_k && active) {
            const double fk = 2.0 * f;
#pragma unroll
            for (int a = 0; a < S::NSA; ++a)
#pragma unroll
                for (int c = 0; c < S::NSC; ++c) {
                    double s = 0.0;
#pragma unroll
                    for (int bq = 0; bq < S::NSB; ++bq)
#pragma unroll
                        for (int d = 0; d < S::NSD; ++d)
                            s += V[(a * S::NSB + bq) * NSCD + c * S::NSD + d] * __ldg(Dm + (long long)(b0 + bq) * M + d0 + d);
                    atomicAdd(Km + (long long)(a0 + a) * M + c0 + c, fk * s);
                }
#pragma unroll
            for (int a = 0; a < S::NSA; ++a)
#pragma unroll
                for (int d = 0; d < S::NSD; ++d) {
                    double s = 0.0;
#pragma unroll
                    for (int bq = 0; bq < S::NSB; ++bq)
#pragma unroll
                        for (int c = 0; c < S::NSC; ++c)
                            s += V[(a * S::NSB + bq) * NSCD + c * S::NSD + d] * __ldg(Dm + (long long)(b0 + bq) * M + c0 + c);
                    atomicAdd(Km + (long long)(a0 + a) * M + d0 + d, fk * s);
                }
#pragma unroll
            for (int bq = 0; bq < S::NSB; ++bq)
#pragma unroll
                for (int c = 0; c < S::NSC; ++c) {
                    double s = 0.0;
#pragma unroll
                    for (int a = 0; a < S::NSA; ++a)
#pragma unroll
                        for (int d = 0; d < S::NSD; ++d)
                            s += V[(a * S::NSB + bq) * NSCD + c * S::NSD + d] * __ldg(Dm + (long long)(a0 + a) * M + d0 + d);
                    atomicAdd(Km + (long long)(b0 + bq) * M + c0 + c, fk * s);
                }
#pragma unroll
            for (int bq = 0; bq < S::NSB; ++bq)
#pragma unroll
                for (int d = 0; d < S::NSD; ++d) {
                    double s = 0.0;
#pragma unroll
                    for (int a = 0; a < S::NSA; ++a)
#pragma unroll
                        for (int c = 0; c < S::NSC; ++c)
                            s += V[(a * S::NSB + bq) * NSCD + c * S::NSD + d] * __ldg(Dm + (long long)(a0 + a) * M + c0 + c);
                    atomicAdd(Km + (long long)(b0 + bq) * M + d0 + d, fk * s);
                }
        }
    }
}

}  // namespace dev
}  // namespace tlno_gpu
