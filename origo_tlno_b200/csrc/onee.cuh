// One-electron overlap, kinetic and nuclear-attraction integrals.
//
// One warp per screened shell pair (A, B), L_A >= L_B, with its Cartesian
// S, T, V blocks in shared memory:
//  * S and T: each lane owns Cartesian component pairs and walks the
//    primitive pairs with the Obara-Saika 1-D shape tables extended to
//    l_b + 2, kinetic 1-D factor
//    T_x = b(2l_b+1) S(l_a,l_b) - 2b^2 S(l_a,l_b+2) - l_b(l_b-1)/2 S(l_a,l_b-2)
//    (reference: integrals/one_electron/onee_integrals.cpp:32-51, 284-416);
//  * V: per primitive pair each lane takes a strided subset of the nuclei,
//    forms the Boys seeds (-2p)^n F_n(p |P-C|^2) and the McMurchie-Davidson
//    R_tuv recursion (unrolled per total order, in registers) and sums
//    Z_K R_tuv; the warp reduces the sums once, three lanes build the
//    Hermite expansion coefficients E^t_ij of the three axes, and the lanes,
//    now owning component pairs, contract them (onee_integrals.cpp:53-157,
//    477-887);
//  * the Cartesian blocks are transformed to real spherical harmonics and
//    written to both triangles of the M x M outputs
//    (onee_matrices.cpp:226-309, 554-607).
// Primitive pairs whose nuclear monopole estimate
// (2 pi / p) e^{-mu AB^2} max|c_a| max|c_b| falls below eps / sum|Z| skip V
// (onee_integrals.cpp:541-546, 638).
#pragma once

#include "device_common.cuh"
#include "launch_types.hpp"

namespace tlno_gpu {
namespace dev {

constexpr int kOneeMaxCart = 15;   // L <= 4

__device__ __forceinline__ double ang_norm(int lx, int ly, int lz) {
    double df = 1.0;
    for (int k = 2 * lx - 1; k > 0; k -= 2) df *= k;
    for (int k = 2 * ly - 1; k > 0; k -= 2) df *= k;
    for (int k = 2 * lz - 1; k > 0; k -= 2) df *= k;
    return 1.0 / sqrt(df);
}

// 1-D overlap shape table S[ia * ncol + ib], ia <= la + lbe, ib <= lbe.
__device__ __forceinline__ void shape_table(double* S, int la, int lbe, double pa, double ab,
                                            double inv2p) {
    const int ltot = la + lbe, ncol = lbe + 1;
    S[0] = 1.0;
    if (ltot >= 1) S[ncol] = pa;
    for (int n = 1; n < ltot; ++n) S[(n + 1) * ncol] = pa * S[n * ncol] + (n * inv2p) * S[(n - 1) * ncol];
    for (int ib = 0; ib < lbe; ++ib)
        for (int ia = 0; ia <= ltot - ib - 1; ++ia)
            S[ia * ncol + ib + 1] = S[(ia + 1) * ncol + ib] + ab * S[ia * ncol + ib];
}

// Hermite expansion coefficients E[(i * (lb+1) + j) * nt + t], nt = la+lb+1.
__device__ __forceinline__ void hermite_table(double* E, int la, int lb, double qx, double alpha,
                                              double beta, double inv2p, double e0) {
    const int ltot = la + lb, nt = ltot + 1, col = lb + 1;
    const double invp = 2.0 * inv2p;
    const double pa = -beta * qx * invp, pb = alpha * qx * invp;
    // work table over ia <= ltot for the bra transfer
    double W[(2 * kMaxL + 1) * (kMaxL + 1) * (2 * kMaxL + 1)];
    const int wcol = col;
    for (int i = 0; i < (ltot + 1) * wcol * nt; ++i) W[i] = 0.0;
    W[0] = e0;
    for (int ia = 0; ia < ltot; ++ia)
        for (int t = 0; t <= ia + 1; ++t) {
            double v = pa * W[(ia * wcol) * nt + t];
            if (t > 0) v += inv2p * W[(ia * wcol) * nt + t - 1];
            if (t < ia) v += (t + 1.0) * W[(ia * wcol) * nt + t + 1];
            W[((ia + 1) * wcol) * nt + t] = v;
        }
    for (int ib = 0; ib < lb; ++ib)
        for (int ia = 0; ia <= ltot; ++ia) {
            const int tmax = min(ia + ib + 1, ltot);
            for (int t = 0; t <= tmax; ++t) {
                double v = pb * W[(ia * wcol + ib) * nt + t];
                if (t > 0) v += inv2p * W[(ia * wcol + ib) * nt + t - 1];
                if (t < ia + ib) v += (t + 1.0) * W[(ia * wcol + ib) * nt + t + 1];
                W[(ia * wcol + ib + 1) * nt + t] = v;
            }
        }
    for (int ia = 0; ia <= la; ++ia)
        for (int ib = 0; ib <= lb; ++ib)
            for (int t = 0; t <= ltot; ++t) E[(ia * col + ib) * nt + t] = W[(ia * wcol + ib) * nt + t];
}

// (-2p)^n F_n(x) for n <= maxn <= 8, evaluated per order as the reference's
// low-order batch does (core/math/general_math.cpp:243-309): a 6-term Taylor
// expansion about the nearest 0.01 node below x = 40; above, erf plus upward
// recursion until x >= 40 + 2 maxn, then the pure asymptotic form.
__device__ __forceinline__ void boys_seeds(int maxn, double x, double p, double* out) {
    if (x < 40.0) {
        const int grid = static_cast<int>(x * 100.0 + 0.5);
        const double d = grid * 0.01 - x;
        const double* row = c_tabs.boys + grid * 40;
        double power = 1.0;
        for (int n = 0; n <= maxn; ++n) {
            double v = row[n + 5];
            for (int k = 4; k >= 0; --k) v = fma(v, d * (1.0 / (k + 1)), row[n + k]);
            out[n] = v * power;
            power *= -2.0 * p;
        }
        return;
    }
    double v = 0.5 * sqrt(3.141592653589793238462643383279502884 / x);
    if (x < 40.0 + 2 * maxn) {
        v *= erf(sqrt(x));
        const double ex = exp(-x), inv2x = 0.5 / x;
        double power = 1.0;
        out[0] = v;
        for (int n = 1; n <= maxn; ++n) {
            v = ((2 * n - 1) * v - ex) * inv2x;
            power *= -2.0 * p;
            out[n] = v * power;
        }
    } else {
        const double factor = -p / x;
        out[0] = v;
        for (int n = 1; n <= maxn; ++n) {
            v *= factor * (2 * n - 1);
            out[n] = v;
        }
    }
}

// Per-warp shared memory of the one-electron kernel (doubles): the Cartesian
// S, T, V blocks, the nucleus-summed R_tuv and the three Hermite tables.
constexpr int kOneeBlk = kOneeMaxCart * kOneeMaxCart;
constexpr int kOneeEAxis = (kMaxL + 1) * (kMaxL + 1) * (2 * kMaxL + 1);
constexpr int kOneeWarpWords = 3 * kOneeBlk + kNCartCum8 + 3 * kOneeEAxis + 1;  // 16-byte multiple

// sum_K Z_K R^{(0)}_{tuv}(P - C_K) over this lane's nuclei for total order LT
// (compile-time, in registers), reduced over the warp into
// Rw[cart_flat(t, u, v)].  Downward recursion in n of
// R^{(n)}_{t,u,v} = X R^{(n+1)}_{t-1,u,v} + (t-1) R^{(n+1)}_{t-2,u,v} (and the
// same in u, v), seeded by R^{(n)}_{000} = (-2p)^n F_n(p |P-C|^2)
// (onee_integrals.cpp:108-157), done in place: within a level the orders are
// visited from the highest down, so every entry of the next level is read
// before it is overwritten.
template <int LT>
__device__ __forceinline__ void nuclear_r_sum(const OneeLaunch& L, double Px, double Py, double Pz, double p,
                                              int lane, double* Rw) {
    constexpr int NR = (LT + 1) * (LT + 2) * (LT + 3) / 6;
    double acc[NR];
#pragma unroll
    for (int r = 0; r < NR; ++r) acc[r] = 0.0;
    for (int K = lane; K < L.n_nuc; K += 32) {
        const double cx = Px - L.nuc[4 * K], cy = Py - L.nuc[4 * K + 1], cz = Pz - L.nuc[4 * K + 2];
        const double Zk = L.nuc[4 * K + 3];
        double F[LT + 1];
        boys_seeds(LT, p * (cx * cx + cy * cy + cz * cz), p, F);
        double R[NR];
        R[0] = F[LT];
#pragma unroll
        for (int n = LT - 1; n >= 0; --n) {
#pragma unroll
            for (int tot = LT - n; tot >= 1; --tot) {
#pragma unroll
                for (int t = tot; t >= 0; --t) {
#pragma unroll
                    for (int u = tot - t; u >= 0; --u) {
                        const int v = tot - t - u;
                        double val;
                        if (t > 0)
                            val = cx * R[cart_flat(t - 1, u, v)] + (t > 1 ? (t - 1) * R[cart_flat(t - 2, u, v)] : 0.0);
                        else if (u > 0)
                            val = cy * R[cart_flat(t, u - 1, v)] + (u > 1 ? (u - 1) * R[cart_flat(t, u - 2, v)] : 0.0);
                        else
                            val = cz * R[cart_flat(t, u, v - 1)] + (v > 1 ? (v - 1) * R[cart_flat(t, u, v - 2)] : 0.0);
                        R[cart_flat(t, u, v)] = val;
                    }
                }
            }
            R[0] = F[n];
        }
#pragma unroll
        for (int r = 0; r < NR; ++r) acc[r] += Zk * R[r];
    }
#pragma unroll
    for (int r = 0; r < NR; ++r) {
        double v = acc[r];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) Rw[r] = v;
    }
}

// The same for total orders above 4 (pairs with f or g shells), with the
// recursion levels in per-thread arrays.
__device__ __noinline__ void nuclear_r_sum_any(const OneeLaunch& L, int ltot, double Px, double Py, double Pz,
                                               double p, int lane, double* Rw) {
    const int nR = ncart_cum(ltot);
    double Rs[kNCartCum8], R0[kNCartCum8], R1[kNCartCum8];
    double F[2 * kMaxL + 1];
    for (int r = 0; r < nR; ++r) Rs[r] = 0.0;
    for (int K = lane; K < L.n_nuc; K += 32) {
        const double cx = Px - L.nuc[4 * K], cy = Py - L.nuc[4 * K + 1], cz = Pz - L.nuc[4 * K + 2];
        const double Zk = L.nuc[4 * K + 3];
        boys_seeds(ltot, p * (cx * cx + cy * cy + cz * cz), p, F);
        double* cur = R0;
        double* nxt = R1;
        for (int n = ltot; n >= 0; --n) {
            const int lim = ltot - n;
            cur[0] = F[n];
            for (int tot = 1; tot <= lim; ++tot)
                for (int t = tot; t >= 0; --t)
                    for (int u = tot - t; u >= 0; --u) {
                        const int v = tot - t - u;
                        double val;
                        if (t > 0) val = cx * nxt[cart_flat(t - 1, u, v)] + (t > 1 ? (t - 1) * nxt[cart_flat(t - 2, u, v)] : 0.0);
                        else if (u > 0) val = cy * nxt[cart_flat(t, u - 1, v)] + (u > 1 ? (u - 1) * nxt[cart_flat(t, u - 2, v)] : 0.0);
                        else val = cz * nxt[cart_flat(t, u, v - 1)] + (v > 1 ? (v - 1) * nxt[cart_flat(t, u, v - 2)] : 0.0);
                        cur[cart_flat(t, u, v)] = val;
                    }
            double* tmp = cur; cur = nxt; nxt = tmp;
        }
        for (int r = 0; r < nR; ++r) Rs[r] += Zk * nxt[r];
    }
    for (int r = 0; r < nR; ++r) {
        double v = Rs[r];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) Rw[r] = v;
    }
}

__global__ void __launch_bounds__(128) onee_kernel(OneeLaunch L) {
    extern __shared__ double onee_smem[];
    const int warps = blockDim.x >> 5;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double* Sc = onee_smem + warp * kOneeWarpWords;  // Cartesian S block [ca * ncb + cb]
    double* Tc = Sc + kOneeBlk;
    double* Vc = Tc + kOneeBlk;
    double* Rw = Vc + kOneeBlk;                       // nucleus-summed R_tuv
    double* Ew = Rw + kNCartCum8;                     // Hermite tables, one per axis
    for (int pi = blockIdx.x * warps + warp; pi < L.n_pairs; pi += gridDim.x * warps) {
        const OneePair pr = L.pairs[pi];
        const int A = pr.A, B = pr.B;
        const int la = L.shell_L[A], lb = L.shell_L[B];
        const int nca = ncart(la), ncb = ncart(lb);
        const double* xa = L.shell_xyz + 3 * A;
        const double* xb = L.shell_xyz + 3 * B;
        const double ab[3] = {xa[0] - xb[0], xa[1] - xb[1], xa[2] - xb[2]};
        const double ab2 = ab[0] * ab[0] + ab[1] * ab[1] + ab[2] * ab[2];
        const int npa = L.shell_nprim[A], npb = L.shell_nprim[B];
        const int pa0 = L.shell_prim[A], pb0 = L.shell_prim[B];
        const int offa = cart_offset(la), offb = cart_offset(lb);
        const int ncomp = nca * ncb;
        for (int cc = lane; cc < ncomp; cc += 32) {
            Sc[cc] = 0.0;
            Tc[cc] = 0.0;
            Vc[cc] = 0.0;
        }
        // ---- overlap and kinetic: lanes own component pairs ----
        if (pr.do_st) {
            for (int cc = lane; cc < ncomp; cc += 32) {
                const int ca = cc / ncb, cb = cc % ncb;
                const int ax = c_cart.xyz[offa + ca][0], ay = c_cart.xyz[offa + ca][1], az = c_cart.xyz[offa + ca][2];
                const int bx = c_cart.xyz[offb + cb][0], by = c_cart.xyz[offb + cb][1], bz = c_cart.xyz[offb + cb][2];
                double s_acc = 0.0, t_acc = 0.0;
                const int lbe = lb + 2, ncol = lbe + 1;
                double Sx[(2 * kMaxL + 3) * (kMaxL + 3)], Sy[(2 * kMaxL + 3) * (kMaxL + 3)], Sz[(2 * kMaxL + 3) * (kMaxL + 3)];
                const double* cfa = L.comp_coef + L.comp_off[A] + ca * npa;
                const double* cfb = L.comp_coef + L.comp_off[B] + cb * npb;
                for (int ia = 0; ia < npa; ++ia) {
                    const double alpha = L.exps[pa0 + ia];
                    const double da = cfa[ia];
                    for (int ib = 0; ib < npb; ++ib) {
                        const double beta = L.exps[pb0 + ib];
                        const double db = cfb[ib];
                        const double p = alpha + beta, invp = 1.0 / p;
                        const double chi = alpha * beta * invp;
                        const double pip = 3.141592653589793238462643383279502884 * invp;
                        const double sss = pip * sqrt(pip) * exp(-chi * ab2);
                        if (la == 0 && lb == 0) {
                            // s-s closed form (onee_integrals.cpp:318-348)
                            const double kin = sss * chi * (3.0 - 2.0 * chi * ab2);
                            s_acc += da * db * sss;
                            t_acc += da * db * kin;
                            continue;
                        }
                        const double inv2p = 0.5 * invp;
                        const double Px = (alpha * xa[0] + beta * xb[0]) * invp;
                        const double Py = (alpha * xa[1] + beta * xb[1]) * invp;
                        const double Pz = (alpha * xa[2] + beta * xb[2]) * invp;
                        shape_table(Sx, la, lbe, Px - xa[0], ab[0], inv2p);
                        shape_table(Sy, la, lbe, Py - xa[1], ab[1], inv2p);
                        shape_table(Sz, la, lbe, Pz - xa[2], ab[2], inv2p);
                        const double w = da * db * sss;
                        const double sx = Sx[ax * ncol + bx], sy = Sy[ay * ncol + by], sz = Sz[az * ncol + bz];
                        s_acc += w * sx * sy * sz;
                        const double tx = beta * (2.0 * bx + 1.0) * sx - 2.0 * beta * beta * Sx[ax * ncol + bx + 2] -
                                          (bx >= 2 ? 0.5 * static_cast<double>(bx * (bx - 1)) * Sx[ax * ncol + bx - 2] : 0.0);
                        const double ty = beta * (2.0 * by + 1.0) * sy - 2.0 * beta * beta * Sy[ay * ncol + by + 2] -
                                          (by >= 2 ? 0.5 * static_cast<double>(by * (by - 1)) * Sy[ay * ncol + by - 2] : 0.0);
                        const double tz = beta * (2.0 * bz + 1.0) * sz - 2.0 * beta * beta * Sz[az * ncol + bz + 2] -
                                          (bz >= 2 ? 0.5 * static_cast<double>(bz * (bz - 1)) * Sz[az * ncol + bz - 2] : 0.0);
                        t_acc += w * (tx * sy * sz + sx * ty * sz + sx * sy * tz);
                    }
                }
                Sc[cc] = s_acc;
                Tc[cc] = t_acc;
            }
        }
        // ---- nuclear attraction: lanes own nuclei, then component pairs ----
        if (pr.do_v) {
            const int ltot = la + lb;
            const int nt = ltot + 1, col = lb + 1;
            double v00 = 0.0;  // s-s: this lane's share
            for (int ia = 0; ia < npa; ++ia) {
                const double alpha = L.exps[pa0 + ia];
                for (int ib = 0; ib < npb; ++ib) {
                    const double beta = L.exps[pb0 + ib];
                    const double p = alpha + beta, invp = 1.0 / p;
                    const double chi = alpha * beta * invp;
                    const double emc = exp(-chi * ab2);
                    const double pip = 3.141592653589793238462643383279502884 * invp;
                    const double screen = 2.0 * pip * emc * L.maxc[pa0 + ia] * L.maxc[pb0 + ib];
                    if (screen < L.screen_thr) continue;
                    const double Px = (alpha * xa[0] + beta * xb[0]) * invp;
                    const double Py = (alpha * xa[1] + beta * xb[1]) * invp;
                    const double Pz = (alpha * xa[2] + beta * xb[2]) * invp;
                    const double neg2pi_over_p = -2.0 * pip;
                    if (ltot == 0) {
                        // s-s: V = d_a d_b (-2 pi / p) e^{-mu AB^2} sum_K Z_K F_0
                        // (onee_integrals.cpp:550-631)
                        double nuc_sum = 0.0;
                        for (int K = lane; K < L.n_nuc; K += 32) {
                            const double cx = Px - L.nuc[4 * K], cy = Py - L.nuc[4 * K + 1], cz = Pz - L.nuc[4 * K + 2];
                            double F0[1];
                            boys_seeds(0, p * (cx * cx + cy * cy + cz * cz), p, F0);
                            nuc_sum += L.nuc[4 * K + 3] * F0[0];
                        }
                        v00 += L.comp_coef[L.comp_off[A] + ia] * L.comp_coef[L.comp_off[B] + ib] *
                               (neg2pi_over_p * emc * nuc_sum);
                        continue;
                    }
                    __syncwarp();  // the previous primitive pair's readers are done
                    switch (ltot) {
                        case 1: nuclear_r_sum<1>(L, Px, Py, Pz, p, lane, Rw); break;
                        case 2: nuclear_r_sum<2>(L, Px, Py, Pz, p, lane, Rw); break;
                        case 3: nuclear_r_sum<3>(L, Px, Py, Pz, p, lane, Rw); break;
                        case 4: nuclear_r_sum<4>(L, Px, Py, Pz, p, lane, Rw); break;
                        default: nuclear_r_sum_any(L, ltot, Px, Py, Pz, p, lane, Rw); break;
                    }
                    const double inv2p = 0.5 * invp;
                    if (lane < 3)
                        hermite_table(Ew + lane * kOneeEAxis, la, lb, ab[lane], alpha, beta, inv2p,
                                      exp(-chi * ab[lane] * ab[lane]));
                    __syncwarp();
                    for (int cc = lane; cc < ncomp; cc += 32) {
                        const int ca = cc / ncb, cb = cc % ncb;
                        const int ax = c_cart.xyz[offa + ca][0], ay = c_cart.xyz[offa + ca][1], az = c_cart.xyz[offa + ca][2];
                        const int bx = c_cart.xyz[offb + cb][0], by = c_cart.xyz[offb + cb][1], bz = c_cart.xyz[offb + cb][2];
                        const double da = L.comp_coef[L.comp_off[A] + ca * npa + ia];
                        const double db = L.comp_coef[L.comp_off[B] + cb * npb + ib];
                        const double* ex = Ew + (ax * col + bx) * nt;
                        const double* ey = Ew + kOneeEAxis + (ay * col + by) * nt;
                        const double* ez = Ew + 2 * kOneeEAxis + (az * col + bz) * nt;
                        double s = 0.0;
                        for (int t = 0; t <= ax + bx; ++t)
                            for (int u = 0; u <= ay + by; ++u) {
                                const double exy = ex[t] * ey[u];
                                for (int v = 0; v <= az + bz; ++v) s += exy * ez[v] * Rw[cart_flat(t, u, v)];
                            }
                        Vc[cc] += (da * db * neg2pi_over_p) * s;
                    }
                }
            }
            if (ltot == 0) {
                for (int o = 16; o > 0; o >>= 1) v00 += __shfl_xor_sync(0xffffffffu, v00, o);
                if (lane == 0) Vc[0] = v00;
            }
        }
        __syncwarp();
        // ---- spherical transform and scatter ----
        const int nsa = nsph(la), nsb = nsph(lb);
        const int a0 = L.shell_sph[A], b0 = L.shell_sph[B];
        const int M = L.M;
        for (int e = lane; e < nsa * nsb; e += 32) {
            const int sa = e / nsb, sb = e % nsb;
            double sv = 0.0, tv = 0.0, vv = 0.0;
            for (int ea = c_c2s.start[la]; ea < c_c2s.start[la] + c_c2s.count[la]; ++ea) {
                if (c_c2s.sph[ea] != sa) continue;
                const int ca = c_c2s.cart[ea];
                const double ka = c_c2s.coef_raw[ea];
                for (int eb = c_c2s.start[lb]; eb < c_c2s.start[lb] + c_c2s.count[lb]; ++eb) {
                    if (c_c2s.sph[eb] != sb) continue;
                    const double k = ka * c_c2s.coef_raw[eb];
                    const int idx = ca * ncb + c_c2s.cart[eb];
                    sv += k * Sc[idx];
                    tv += k * Tc[idx];
                    vv += k * Vc[idx];
                }
            }
            const long long ij = (long long)(a0 + sa) * M + b0 + sb;
            const long long ji = (long long)(b0 + sb) * M + a0 + sa;
            if (pr.do_st) { L.S[ij] = sv; L.S[ji] = sv; L.T[ij] = tv; L.T[ji] = tv; }
            if (pr.do_v) { L.V[ij] = vv; L.V[ji] = vv; }
        }
        __syncwarp();
    }
}

}  // namespace dev
}  // namespace tlno_gpu
