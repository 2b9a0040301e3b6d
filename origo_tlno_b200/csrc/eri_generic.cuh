// Generic warp-per-quartet Rys ERI kernel (any class up to (gg|gg)).
//
// One warp evaluates one contracted shell quartet (AB|CD):
//  1. the (primitive pair x primitive pair x root) items are spread over the
//     lanes, 32 at a time; each lane builds the three 2-D Rys integral tables
//     G_x, G_y, G_z(i <= La+Lb, k <= Lc+Ld) of its item by the vertical
//     recurrences of the reference (rys_engine.ipp:13704-13715, 12694-12749)
//     into its shared-memory slot, with the quadrature weight and the
//     2 pi^{5/2} w_ab w_cd / sqrt(p+q) prefactor folded into G_z;
//  2. each lane owns a disjoint set of contracted radial integrals
//     (a0|c0), |a| in [La, La+Lb], |c| in [Lc, Lc+Ld], and accumulates
//     sum_items Gx Gy Gz for them (rys_engine.ipp:13616-13627);
//  3. the horizontal transfer and the Cartesian->spherical projection are
//     applied together as two small dense maps built on the fly from AB and
//     CD, (a b| = sum_u C(b,u) (A-B)^{b-u} (a+u 0| per axis, with the
//     normalised spherical coefficients folded in (the radial projector form
//     of rys_engine.ipp:18370-18430);
//  4. the spherical block is either stored (ERI oracle endpoint), reduced to
//     the Schwarz bound (diagonal quartets), or digested into J and K.
#pragma once

#include "eri_common.cuh"

namespace tlno_gpu {
namespace dev {

constexpr int kGenericBatch = 32;

struct GenericLayout {
    int las, lcs;        // La+Lb, Lc+Ld
    int ks, gs;          // k stride (Lc+Ld+1), per-axis G size
    int gslot;           // doubles per item slot: 3 gs rounded up to odd (conflict-free per-lane slots)
    int nas, ncs;        // radial slice sizes
    int nsab, nscd;      // spherical pair sizes
    int na, nb, nc, nd;  // spherical sizes per shell
    // offsets in doubles within the warp's region
    int off_T, off_PB, off_PK, off_X, off_V, off_P;
    int words;           // doubles per warp
    __host__ __device__ void init(int la, int lb, int lc, int ld) {
        las = la + lb;
        lcs = lc + ld;
        ks = lcs + 1;
        gs = (las + 1) * ks;
        nas = ncart_cum(las) - cart_offset(la);
        ncs = ncart_cum(lcs) - cart_offset(lc);
        na = nsph(la); nb = nsph(lb); nc = nsph(lc); nd = nsph(ld);
        nsab = na * nb;
        nscd = nc * nd;
        gslot = (3 * gs) | 1;
        const int g_words = kGenericBatch * gslot;
        off_X = 0;
        off_V = off_X + nas * nscd;
        off_P = off_V + nsab * nscd;
        const int p_words = na * nb + nc * nd + nb * nd + nb * nc + na * nd + na * nc;
        int tail = off_P + p_words;
        int region0 = g_words > tail ? g_words : tail;
        off_T = region0;
        off_PB = off_T + nas * ncs;
        off_PK = off_PB + nsab * nas;
        words = off_PK + nscd * ncs;
        words = (words + 1) & ~1;  // 16-byte multiple
    }
};

template <typename R>
__device__ __forceinline__ void vrr_2d(R* G, int las, int lcs, int ks, R c00, R d00,
                                       R b00, R b10, R b01, R seed) {
    G[0] = seed;
    if (las > 0) {
        G[ks] = c00 * seed;
        for (int i = 1; i < las; ++i)
            G[(i + 1) * ks] = c00 * G[i * ks] + R(i) * b10 * G[(i - 1) * ks];
    }
    for (int k = 0; k < lcs; ++k) {
        for (int i = 0; i <= las; ++i) {
            R v = d00 * G[i * ks + k];
            if (i > 0) v += R(i) * b00 * G[(i - 1) * ks + k];
            if (k > 0) v += R(k) * b01 * G[i * ks + k - 1];
            G[i * ks + k + 1] = v;
        }
    }
}

// Builds the dense (HRR + spherical) projector for one shell pair: element
// (s_ab, flat(a') - off(la)), |a'| in [la, la+lb], at Pm[s_ab * rs + col * cs]
// (rs = nslice, cs = 1: row-major; rs = 1, cs = rows: transposed).
__device__ __forceinline__ void build_pair_projector(double* Pm, int la, int lb,
                                                     double abx, double aby, double abz,
                                                     int lane, bool transposed = false) {
    const int na = nsph(la), nb = nsph(lb);
    const int nslice = ncart_cum(la + lb) - cart_offset(la);
    const int off_a = cart_offset(la), off_b = cart_offset(lb);
    const int rs = transposed ? 1 : nslice, cs = transposed ? na * nb : 1;
    const double ab[3] = {abx, aby, abz};
    for (int row = lane; row < na * nb; row += 32) {
        double* out = Pm + row * rs;
        for (int c = 0; c < nslice; ++c) out[c * cs] = 0.0;
        const int sa = row / nb, sb = row % nb;
        for (int ea = c_c2s.start[la]; ea < c_c2s.start[la] + c_c2s.count[la]; ++ea) {
            if (c_c2s.sph[ea] != sa) continue;
            const int ca = off_a + c_c2s.cart[ea];
            const int ax = c_cart.xyz[ca][0], ay = c_cart.xyz[ca][1], az = c_cart.xyz[ca][2];
            const double ka = c_c2s.coef[ea];
            for (int eb = c_c2s.start[lb]; eb < c_c2s.start[lb] + c_c2s.count[lb]; ++eb) {
                if (c_c2s.sph[eb] != sb) continue;
                const int cb = off_b + c_c2s.cart[eb];
                const int bxyz[3] = {c_cart.xyz[cb][0], c_cart.xyz[cb][1], c_cart.xyz[cb][2]};
                const double kab = ka * c_c2s.coef[eb];
                // binomial expansion per axis
                double fx[5], fy[5], fz[5];
                const int* bb = bxyz;
                double* f3[3] = {fx, fy, fz};
                for (int ax3 = 0; ax3 < 3; ++ax3) {
                    const int b = bb[ax3];
                    // C(b,u) * ab^(b-u)
                    double binom = 1.0;
                    for (int u = 0; u <= b; ++u) {
                        double pw = 1.0;
                        for (int e = 0; e < b - u; ++e) pw *= ab[ax3];
                        f3[ax3][u] = binom * pw;
                        binom = binom * (b - u) / (u + 1);
                    }
                }
                for (int ux = 0; ux <= bxyz[0]; ++ux)
                    for (int uy = 0; uy <= bxyz[1]; ++uy)
                        for (int uz = 0; uz <= bxyz[2]; ++uz) {
                            const int col = cart_flat(ax + ux, ay + uy, az + uz) - off_a;
                            out[col * cs] += kab * fx[ux] * fy[uy] * fz[uz];
                        }
            }
        }
    }
}

// build_pb = false reuses the bra projector this warp built for the same
// bra pair (it lives in its own region of the warp's shared memory).
// jon / kon (J/K mode) are 0 when the density screen drops the quartet's
// Coulomb / exchange contributions.
template <typename R, int MODE>
__device__ void generic_quartet(const PlanView& pv, const ClassLaunch& cl,
                                const GenericLayout& lay, double* wsm, int lane,
                                int bra, int ket, int quartet_id, bool build_pb = true,
                                double jon = 1.0, double kon = 1.0) {
    const int A = pv.pair_A[bra], B = pv.pair_B[bra];
    const int C = pv.pair_A[ket], D = pv.pair_B[ket];
    const double* xa = pv.shell_xyz + 3 * A;
    const double* xb = pv.shell_xyz + 3 * B;
    const double* xc = pv.shell_xyz + 3 * C;
    const double* xd = pv.shell_xyz + 3 * D;
    const int la = cl.la, lb = cl.lb, lc = cl.lc, ld = cl.ld;
    const int nroots = (la + lb + lc + ld) / 2 + 1;
    const int npb = pv.pair_nprim[bra], npk = pv.pair_nprim[ket];
    const DPrimPair* pb = pv.prim + pv.pair_prim_off[bra];
    const DPrimPair* pk = pv.prim + pv.pair_prim_off[ket];
    R* Gs = reinterpret_cast<R*>(wsm);
    R* T = reinterpret_cast<R*>(wsm + lay.off_T);
    const int ntr = lay.nas * lay.ncs;
    for (int e = lane; e < ntr; e += 32) T[e] = R(0);

    const R Ax = R(xa[0]), Ay = R(xa[1]), Az = R(xa[2]);
    const R Cx = R(xc[0]), Cy = R(xc[1]), Cz = R(xc[2]);
    const int n_items = npb * npk * nroots;
    const int gslot = lay.gslot;
    const int offa = cart_offset(la), offc = cart_offset(lc);
    // Primitive FASTSCHWARZ (J/K mode, classes up to f as the reference's
    // shell4 portfolio): a dropped primitive quartet gets a zero seed.
    const bool fs_on = MODE == kJK && cl.fs_thr2 > 0.0 && la <= 3 && lb <= 3 && lc <= 3 && ld <= 3;
    const int pob = pv.pair_prim_off[bra], pok = pv.pair_prim_off[ket];
    __syncwarp();
    for (int base = 0; base < n_items; base += kGenericBatch) {
        const int item = base + lane;
        if (item < n_items) {
            const int r = item % nroots;
            const int pq = item / nroots;
            const int ib = pq / npk, ik = pq - ib * npk;
            const DPrimPair bp = pb[ib];
            const DPrimPair kp = pk[ik];
            const R p = R(bp.p), q = R(kp.p);
            const R pqs = p + q;
            const R inv = R(1) / pqs;
            const R PQx = R(bp.Px) - R(kp.Px), PQy = R(bp.Py) - R(kp.Py), PQz = R(bp.Pz) - R(kp.Pz);
            const R Targ = p * q * inv * (PQx * PQx + PQy * PQy + PQz * PQz);
            R t2, wt;
            if (sizeof(R) == 4 && nroots >= 4) {
                // FP64 carve-out of the FP32 pass: high-L roots and weights
                double t2d, wtd;
                rys_root<double>(nroots, double(Targ), r, t2d, wtd);
                t2 = R(t2d);
                wt = R(wtd);
            } else {
                rys_root<R>(nroots, Targ, r, t2, wt);
            }
            R pref = R(34.98683665524972497) * R(bp.w) * R(kp.w) / sqrt(pqs);
            if (fs_on && !(pv.prim_fs[pob + ib] * pv.prim_fs[pok + ik] >= cl.fs_thr2)) pref = R(0);
            const R qo = q * inv, po = p * inv;
            const R b00 = R(0.5) * inv * t2;
            const R b10 = R(0.5) * R(bp.invp) * (R(1) - qo * t2);
            const R b01 = R(0.5) * R(kp.invp) * (R(1) - po * t2);
            R* g = Gs + lane * gslot;
            vrr_2d<R>(g, lay.las, lay.lcs, lay.ks, (R(bp.Px) - Ax) - qo * PQx * t2,
                      (R(kp.Px) - Cx) + po * PQx * t2, b00, b10, b01, R(1));
            vrr_2d<R>(g + lay.gs, lay.las, lay.lcs, lay.ks, (R(bp.Py) - Ay) - qo * PQy * t2,
                      (R(kp.Py) - Cy) + po * PQy * t2, b00, b10, b01, R(1));
            vrr_2d<R>(g + 2 * lay.gs, lay.las, lay.lcs, lay.ks, (R(bp.Pz) - Az) - qo * PQz * t2,
                      (R(kp.Pz) - Cz) + po * PQz * t2, b00, b10, b01, pref * wt);
        }
        __syncwarp();
        const int nvalid = min(kGenericBatch, n_items - base);
        for (int e = lane; e < ntr; e += 32) {
            const int ia = e / lay.ncs, ic = e - ia * lay.ncs;
            const int fa = offa + ia, fc = offc + ic;
            const int ix = c_cart.xyz[fa][0] * lay.ks + c_cart.xyz[fc][0];
            const int iy = lay.gs + c_cart.xyz[fa][1] * lay.ks + c_cart.xyz[fc][1];
            const int iz = 2 * lay.gs + c_cart.xyz[fa][2] * lay.ks + c_cart.xyz[fc][2];
            R acc = T[e];
            const R* g = Gs;
            for (int s = 0; s < nvalid; ++s, g += gslot) acc += g[ix] * g[iy] * g[iz];
            T[e] = acc;
        }
        __syncwarp();
    }

    // HRR + spherical projection: V = PB * T * PK^T.
    double* PB = wsm + lay.off_PB;
    double* PK = wsm + lay.off_PK;
    if (build_pb) build_pair_projector(PB, la, lb, xa[0] - xb[0], xa[1] - xb[1], xa[2] - xb[2], lane);
    build_pair_projector(PK, lc, ld, xc[0] - xd[0], xc[1] - xd[1], xc[2] - xd[2], lane);
    __syncwarp();
    double* X = wsm + lay.off_X;
    double* V = wsm + lay.off_V;
    for (int e = lane; e < lay.nas * lay.nscd; e += 32) {
        const int ia = e / lay.nscd, s = e - ia * lay.nscd;
        const R* trow = T + ia * lay.ncs;
        const double* prow = PK + s * lay.ncs;
        double acc = 0.0;
        for (int ic = 0; ic < lay.ncs; ++ic) acc += double(trow[ic]) * prow[ic];
        X[e] = acc;
    }
    __syncwarp();
    for (int e = lane; e < lay.nsab * lay.nscd; e += 32) {
        const int sab = e / lay.nscd, s = e - sab * lay.nscd;
        const double* prow = PB + sab * lay.nas;
        double acc = 0.0;
        for (int ia = 0; ia < lay.nas; ++ia) acc += prow[ia] * X[ia * lay.nscd + s];
        V[e] = acc;
    }
    __syncwarp();

    if (MODE == kStore) {
        double* out = cl.out + cl.out_off[quartet_id];
        for (int e = lane; e < lay.nsab * lay.nscd; e += 32) out[e] = V[e];
    } else if (MODE == kSchwarz) {
        double m = 0.0;
        for (int s = lane; s < lay.nsab; s += 32) m = fmax(m, V[s * lay.nscd + s]);
        for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
        if (lane == 0) {
            double q = sqrt(m * (1.0 + 64.0 * 2.220446049250313e-16));
            if (q > 0.0) q = nextafter(q, 1e300);
            cl.out[quartet_id] = q;
        }
    } else {
        // J/K digestion with shell-level degeneracy f (8-fold symmetry):
        // J[ab] += 4f V P[cd], J[cd] += 4f V P[ab], K[ac] += 2f V P[bd],
        // K[ad] += 2f V P[bc], K[bc] += 2f V P[ad], K[bd] += 2f V P[ac];
        // the final pass symmetrises (X + X^T)/2 (consumer_policies.ipp:87-157,
        // direct_build.ipp:471-482 for the same algebra at AO level).
        if (cl.checksum) {
            // ERI checksum stream: canonical unique elements of the block
            const int a0 = pv.shell_sph[A], b0 = pv.shell_sph[B];
            const int c0 = pv.shell_sph[C], d0 = pv.shell_sph[D];
            double s = 0.0;
            for (int e = lane; e < lay.nsab * lay.nscd; e += 32) {
                const int sab = e / lay.nscd, scd = e - sab * lay.nscd;
                if (canonical_element(A == B, C == D, bra == ket, a0, sab / lay.nb, b0, sab % lay.nb, c0,
                                      scd / lay.nd, d0, scd % lay.nd))
                    s += V[e];
            }
            for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            if (lane == 0 && s != 0.0) atomicAdd(cl.checksum, s);
            __syncwarp();
            return;
        }
        const int mol = pv.pair_mol ? pv.pair_mol[bra] : 0;
        const int M = pv.mol_M ? pv.mol_M[mol] : cl.M;
        const long long mbase = pv.mol_mat_off ? pv.mol_mat_off[mol] : 0;
        const double* Dm = cl.dens + mbase;
        double* Jm = cl.J + mbase;
        double* Km = cl.K + mbase;
        const int a0 = pv.shell_sph[A], b0 = pv.shell_sph[B];
        const int c0 = pv.shell_sph[C], d0 = pv.shell_sph[D];
        double f = 1.0;
        if (A == B) f *= 0.5;
        if (C == D) f *= 0.5;
        if (bra == ket) f *= 0.5;
        const int na = lay.na, nb = lay.nb, nc = lay.nc, nd = lay.nd;
        double* Pab = wsm + lay.off_P;
        double* Pcd = Pab + na * nb;
        double* Pbd = Pcd + nc * nd;
        double* Pbc = Pbd + nb * nd;
        double* Pad = Pbc + nb * nc;
        double* Pac = Pad + na * nd;
        for (int e = lane; e < na * nb; e += 32) Pab[e] = Dm[(long long)(a0 + e / nb) * M + b0 + e % nb];
        for (int e = lane; e < nc * nd; e += 32) Pcd[e] = Dm[(long long)(c0 + e / nd) * M + d0 + e % nd];
        for (int e = lane; e < nb * nd; e += 32) Pbd[e] = Dm[(long long)(b0 + e / nd) * M + d0 + e % nd];
        for (int e = lane; e < nb * nc; e += 32) Pbc[e] = Dm[(long long)(b0 + e / nc) * M + c0 + e % nc];
        for (int e = lane; e < na * nd; e += 32) Pad[e] = Dm[(long long)(a0 + e / nd) * M + d0 + e % nd];
        for (int e = lane; e < na * nc; e += 32) Pac[e] = Dm[(long long)(a0 + e / nc) * M + c0 + e % nc];
        __syncwarp();
        const int nscd = lay.nscd;
        if (cl.want_j && jon != 0.0) {
            const double fj = 4.0 * f;
            for (int sab = lane; sab < na * nb; sab += 32) {
                double s = 0.0;
                for (int t = 0; t < nscd; ++t) s += V[sab * nscd + t] * Pcd[t];
                atomicAdd(Jm + (long long)(a0 + sab / nb) * M + b0 + sab % nb, fj * s);
            }
            for (int scd = lane; scd < nscd; scd += 32) {
                double s = 0.0;
                for (int t = 0; t < na * nb; ++t) s += V[t * nscd + scd] * Pab[t];
                atomicAdd(Jm + (long long)(c0 + scd / nd) * M + d0 + scd % nd, fj * s);
            }
        }
        if (cl.want_k && kon != 0.0) {
            const double fk = 2.0 * f;
            for (int e = lane; e < na * nc; e += 32) {
                const int a = e / nc, c = e % nc;
                double s = 0.0;
                for (int b = 0; b < nb; ++b)
                    for (int d = 0; d < nd; ++d) s += V[(a * nb + b) * nscd + c * nd + d] * Pbd[b * nd + d];
                atomicAdd(Km + (long long)(a0 + a) * M + c0 + c, fk * s);
            }
            for (int e = lane; e < na * nd; e += 32) {
                const int a = e / nd, d = e % nd;
                double s = 0.0;
                for (int b = 0; b < nb; ++b)
                    for (int c = 0; c < nc; ++c) s += V[(a * nb + b) * nscd + c * nd + d] * Pbc[b * nc + c];
                atomicAdd(Km + (long long)(a0 + a) * M + d0 + d, fk * s);
            }
            for (int e = lane; e < nb * nc; e += 32) {
                const int b = e / nc, c = e % nc;
                double s = 0.0;
                for (int a = 0; a < na; ++a)
                    for (int d = 0; d < nd; ++d) s += V[(a * nb + b) * nscd + c * nd + d] * Pad[a * nd + d];
                atomicAdd(Km + (long long)(b0 + b) * M + c0 + c, fk * s);
            }
            for (int e = lane; e < nb * nd; e += 32) {
                const int b = e / nd, d = e % nd;
                double s = 0.0;
                for (int a = 0; a < na; ++a)
                    for (int c = 0; c < nc; ++c) s += V[(a * nb + b) * nscd + c * nd + d] * Pac[a * nc + c];
                atomicAdd(Km + (long long)(b0 + b) * M + d0 + d, fk * s);
            }
        }
    }
    __syncwarp();
}

// Explicit quartet list (STORE and SCHWARZ modes).
template <typename R, int MODE>
__global__ void eri_generic_list_kernel(PlanView pv, ClassLaunch cl) {
    extern __shared__ double smem[];
    GenericLayout lay;
    lay.init(cl.la, cl.lb, cl.lc, cl.ld);
    const int warps = blockDim.x >> 5;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double* wsm = smem + warp * lay.words;
    for (int q = blockIdx.x * warps + warp; q < cl.n_quartets; q += gridDim.x * warps)
        generic_quartet<R, MODE>(pv, cl, lay, wsm, lane, cl.q_bra[q], cl.q_ket[q], q);
}

// Tiled schedule (J/K mode): tile = 1 bra pair x bk ket pairs.
template <typename R>
__global__ void eri_generic_jk_kernel(PlanView pv, ClassLaunch cl) {
    extern __shared__ double smem[];
    GenericLayout lay;
    lay.init(cl.la, cl.lb, cl.lc, cl.ld);
    const int warps = blockDim.x >> 5;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double* wsm = smem + warp * lay.words;
    const double thr = (cl.prec_mode != 0) ? cl.tau_mix / fmax(*cl.dmax, 1e-300) : 0.0;
    int pb_bra = -1;  // bra pair whose projector this warp holds
    for (int tile = cl.tile_begin + blockIdx.x; tile < cl.tile_end; tile += gridDim.x) {
        const int b = find_block(cl.tile_prefix, cl.n_blocks, tile);
        const int kb = tile - __ldg(cl.tile_prefix + b);
        const BlockDesc bd = cl.blocks[b];
        const int bra = __ldg(cl.bra_list + bd.bra0);  // one bra per block
        const int i = bra - bd.xbeg;
        const double qi = pv.pair_Q[bra];
        for (int jj = warp; jj < cl.bk; jj += warps) {
            const int j = kb * cl.bk + jj;
            if (j >= bd.nket) break;
            if (cl.same && bd.koff + j > i) break;
            const int ket = bd.ket0 + j;
            const double qq = qi * pv.pair_Q[ket];
            if (!(qq >= cl.tau)) continue;
            if (cl.prec_mode == 1 && !(qq >= thr)) continue;
            if (cl.prec_mode == 2 && qq >= thr) continue;
            bool lj = true, lk = true;
            if (cl.den.mode) {
                const int mol = pv.pair_mol ? pv.pair_mol[ket] : 0;
                density_live(cl, pv, mol, pv.pair_A[bra], pv.pair_B[bra], pv.pair_A[ket], pv.pair_B[ket], qq, lj, lk);
                if (!lj && !lk) continue;
            }
            generic_quartet<R, kJK>(pv, cl, lay, wsm, lane, bra, ket, 0, bra != pb_bra, lj ? 1.0 : 0.0,
                                    lk ? 1.0 : 0.0);
            pb_bra = bra;
        }
    }
}

// ---------------------------------------------------------------------------
// CTA-cooperative J/K kernel for the classes the compile-time kernels do not
// cover (two f shells, or deep d/f slices).  One thread block works on one
// contracted quartet at a time, so a class whose radial block, transfer
// products and 2-D tables need tens of KB of shared memory keeps 4-8 warps
// busy per block instead of one warp per block.  The HRR + spherical
// projectors of both pairs come precomputed from the plan (one per shell
// pair, built once per plan by pair_projector_kernel).
//
// Shared memory (doubles): region0 = max(NB item slots x 3 2-D tables,
// X + V + the six density blocks), then the radial block T.
struct GenericCtaLayout {
    int las, lcs, ks, gs, gslot, nas, ncs, na, nb, nc, nd, nsab, nscd;
    int nb_items;  // item slots per batch
    int off_X, off_V, off_P, off_T, words;
    __host__ __device__ void init(int la, int lb, int lc, int ld, int nbi) {
        las = la + lb;
        lcs = lc + ld;
        ks = lcs + 1;
        gs = (las + 1) * ks;
        nas = ncart_cum(las) - cart_offset(la);
        ncs = ncart_cum(lcs) - cart_offset(lc);
        na = nsph(la); nb = nsph(lb); nc = nsph(lc); nd = nsph(ld);
        nsab = na * nb;
        nscd = nc * nd;
        nb_items = nbi;
        // odd slot size: the threads' own slots fall in different banks
        gslot = (3 * gs) | 1;
        const int g_words = nb_items * gslot;
        off_X = 0;
        off_V = off_X + nas * nscd;
        off_P = off_V + nsab * nscd;
        const int tail = off_P + na * nb + nc * nd + nb * nd + nb * nc + na * nd + na * nc;
        off_T = ((g_words > tail ? g_words : tail) + 1) & ~1;
        words = (off_T + nas * ncs + 1) & ~1;
    }
};

// Projector block of one shell pair, stored transposed:
// Pm[(flat(a') - off(la)) * rows + s_ab], rows = (2la+1)(2lb+1), so that the
// threads of a warp, which take consecutive rows, read consecutive words.
__device__ __forceinline__ int pair_projector_words(int la, int lb) {
    return nsph(la) * nsph(lb) * (ncart_cum(la + lb) - cart_offset(la));
}

// Builds the projector of every pair that has an offset (warp per pair).
__global__ void pair_projector_kernel(const int* pair_A, const int* pair_B, const double* shell_xyz,
                                      const int* shell_L, const long long* off, int n_pairs, double* out) {
    const int warps = blockDim.x >> 5;
    const int lane = threadIdx.x & 31;
    for (int k = blockIdx.x * warps + (threadIdx.x >> 5); k < n_pairs; k += gridDim.x * warps) {
        const long long o = off[k];
        if (o < 0) continue;
        const int A = pair_A[k], B = pair_B[k];
        const double* xa = shell_xyz + 3 * A;
        const double* xb = shell_xyz + 3 * B;
        build_pair_projector(out + o, shell_L[A], shell_L[B], xa[0] - xb[0], xa[1] - xb[1], xa[2] - xb[2], lane,
                             true);
    }
}

template <typename R>
__device__ void generic_quartet_cta(const PlanView& pv, const ClassLaunch& cl, const GenericCtaLayout& lay,
                                    double* sm, int bra, int ket, bool jon, bool kon) {
    const int tid = threadIdx.x, nt = blockDim.x;
    const int A = pv.pair_A[bra], B = pv.pair_B[bra];
    const int C = pv.pair_A[ket], D = pv.pair_B[ket];
    const double* xa = pv.shell_xyz + 3 * A;
    const double* xc = pv.shell_xyz + 3 * C;
    const int la = cl.la, lb = cl.lb, lc = cl.lc, ld = cl.ld;
    const int nroots = (la + lb + lc + ld) / 2 + 1;
    const int npb = pv.pair_nprim[bra], npk = pv.pair_nprim[ket];
    const int pob = pv.pair_prim_off[bra], pok = pv.pair_prim_off[ket];
    const DPrimPair* pb = pv.prim + pob;
    const DPrimPair* pk = pv.prim + pok;
    R* Gs = reinterpret_cast<R*>(sm);
    R* T = reinterpret_cast<R*>(sm + lay.off_T);
    const int ntr = lay.nas * lay.ncs;
    for (int e = tid; e < ntr; e += nt) T[e] = R(0);

    const R Ax = R(xa[0]), Ay = R(xa[1]), Az = R(xa[2]);
    const R Cx = R(xc[0]), Cy = R(xc[1]), Cz = R(xc[2]);
    const int n_items = npb * npk * nroots;
    const int gslot = lay.gslot;
    const int offa = cart_offset(la), offc = cart_offset(lc);
    const bool fs_on = cl.fs_thr2 > 0.0 && la <= 3 && lb <= 3 && lc <= 3 && ld <= 3;
    for (int base = 0; base < n_items; base += lay.nb_items) {
        const int item = base + tid;
        if (tid < lay.nb_items && item < n_items) {
            const int r = item % nroots;
            const int pq = item / nroots;
            const int ib = pq / npk, ik = pq - ib * npk;
            const DPrimPair bp = pb[ib];
            const DPrimPair kp = pk[ik];
            const R p = R(bp.p), q = R(kp.p);
            const R pqs = p + q;
            const R inv = R(1) / pqs;
            const R PQx = R(bp.Px) - R(kp.Px), PQy = R(bp.Py) - R(kp.Py), PQz = R(bp.Pz) - R(kp.Pz);
            const R Targ = p * q * inv * (PQx * PQx + PQy * PQy + PQz * PQz);
            R t2, wt;
            if (sizeof(R) == 4 && nroots >= 4) {
                // FP64 carve-out of the FP32 pass: high-L roots and weights
                double t2d, wtd;
                rys_root<double>(nroots, double(Targ), r, t2d, wtd);
                t2 = R(t2d);
                wt = R(wtd);
            } else {
                rys_root<R>(nroots, Targ, r, t2, wt);
            }
            R pref = R(34.98683665524972497) * R(bp.w) * R(kp.w) / sqrt(pqs);
            if (fs_on && !(pv.prim_fs[pob + ib] * pv.prim_fs[pok + ik] >= cl.fs_thr2)) pref = R(0);
            const R qo = q * inv, po = p * inv;
            const R b00 = R(0.5) * inv * t2;
            const R b10 = R(0.5) * R(bp.invp) * (R(1) - qo * t2);
            const R b01 = R(0.5) * R(kp.invp) * (R(1) - po * t2);
            R* g = Gs + tid * gslot;
            vrr_2d<R>(g, lay.las, lay.lcs, lay.ks, (R(bp.Px) - Ax) - qo * PQx * t2,
                      (R(kp.Px) - Cx) + po * PQx * t2, b00, b10, b01, R(1));
            vrr_2d<R>(g + lay.gs, lay.las, lay.lcs, lay.ks, (R(bp.Py) - Ay) - qo * PQy * t2,
                      (R(kp.Py) - Cy) + po * PQy * t2, b00, b10, b01, R(1));
            vrr_2d<R>(g + 2 * lay.gs, lay.las, lay.lcs, lay.ks, (R(bp.Pz) - Az) - qo * PQz * t2,
                      (R(kp.Pz) - Cz) + po * PQz * t2, b00, b10, b01, pref * wt);
        }
        __syncthreads();
        const int nvalid = min(lay.nb_items, n_items - base);
        for (int e = tid; e < ntr; e += nt) {
            const int ia = e / lay.ncs, ic = e - ia * lay.ncs;
            const int fa = offa + ia, fc = offc + ic;
            const int ix = c_cart.xyz[fa][0] * lay.ks + c_cart.xyz[fc][0];
            const int iy = lay.gs + c_cart.xyz[fa][1] * lay.ks + c_cart.xyz[fc][1];
            const int iz = 2 * lay.gs + c_cart.xyz[fa][2] * lay.ks + c_cart.xyz[fc][2];
            R acc = T[e];
            const R* g = Gs;
            for (int s = 0; s < nvalid; ++s, g += gslot) acc += g[ix] * g[iy] * g[iz];
            T[e] = acc;
        }
        __syncthreads();
    }

    // HRR + spherical projection with the plan's (transposed) pair
    // projectors: X = T PK^T, V = PB X.  Consecutive threads take
    // consecutive ket rows s (coalesced PK reads) and share the bra row.
    const double* PBt = pv.proj + pv.proj_off[bra];
    const double* PKt = pv.proj + pv.proj_off[ket];
    double* X = sm + lay.off_X;
    double* V = sm + lay.off_V;
    for (int e = tid; e < lay.nas * lay.nscd; e += nt) {
        const int ia = e / lay.nscd, s = e - ia * lay.nscd;
        const R* trow = T + ia * lay.ncs;
        double acc = 0.0;
        for (int ic = 0; ic < lay.ncs; ++ic) acc += double(trow[ic]) * __ldg(PKt + ic * lay.nscd + s);
        X[e] = acc;
    }
    __syncthreads();
    for (int e = tid; e < lay.nsab * lay.nscd; e += nt) {
        const int sab = e / lay.nscd, s = e - sab * lay.nscd;
        double acc = 0.0;
        for (int ia = 0; ia < lay.nas; ++ia) acc += __ldg(PBt + ia * lay.nsab + sab) * X[ia * lay.nscd + s];
        V[e] = acc;
    }
    __syncthreads();

    if (cl.checksum) {
        // ERI checksum stream: canonical unique elements of the block
        const int a0 = pv.shell_sph[A], b0 = pv.shell_sph[B];
        const int c0 = pv.shell_sph[C], d0 = pv.shell_sph[D];
        double s = 0.0;
        for (int e = tid; e < lay.nsab * lay.nscd; e += nt) {
            const int sab = e / lay.nscd, scd = e - sab * lay.nscd;
            if (canonical_element(A == B, C == D, bra == ket, a0, sab / lay.nb, b0, sab % lay.nb, c0,
                                  scd / lay.nd, d0, scd % lay.nd))
                s += V[e];
        }
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if ((tid & 31) == 0 && s != 0.0) atomicAdd(cl.checksum, s);
        __syncthreads();
        return;
    }
    // J/K digestion with shell-level degeneracy f (consumer_policies.ipp:87-157)
    const int mol = pv.pair_mol ? pv.pair_mol[bra] : 0;
    const int M = pv.mol_M ? pv.mol_M[mol] : cl.M;
    const long long mbase = pv.mol_mat_off ? pv.mol_mat_off[mol] : 0;
    const double* Dm = cl.dens + mbase;
    double* Jm = cl.J + mbase;
    double* Km = cl.K + mbase;
    const int a0 = pv.shell_sph[A], b0 = pv.shell_sph[B];
    const int c0 = pv.shell_sph[C], d0 = pv.shell_sph[D];
    double f = 1.0;
    if (A == B) f *= 0.5;
    if (C == D) f *= 0.5;
    if (bra == ket) f *= 0.5;
    const int na = lay.na, nb = lay.nb, nc = lay.nc, nd = lay.nd;
    double* Pab = sm + lay.off_P;
    double* Pcd = Pab + na * nb;
    double* Pbd = Pcd + nc * nd;
    double* Pbc = Pbd + nb * nd;
    double* Pad = Pbc + nb * nc;
    double* Pac = Pad + na * nd;
    for (int e = tid; e < na * nb; e += nt) Pab[e] = Dm[(long long)(a0 + e / nb) * M + b0 + e % nb];
    for (int e = tid; e < nc * nd; e += nt) Pcd[e] = Dm[(long long)(c0 + e / nd) * M + d0 + e % nd];
    for (int e = tid; e < nb * nd; e += nt) Pbd[e] = Dm[(long long)(b0 + e / nd) * M + d0 + e % nd];
    for (int e = tid; e < nb * nc; e += nt) Pbc[e] = Dm[(long long)(b0 + e / nc) * M + c0 + e % nc];
    for (int e = tid; e < na * nd; e += nt) Pad[e] = Dm[(long long)(a0 + e / nd) * M + d0 + e % nd];
    for (int e = tid; e < na * nc; e += nt) Pac[e] = Dm[(long long)(a0 + e / nc) * M + c0 + e % nc];
    __syncthreads();
    const int nscd = lay.nscd;
    if (cl.want_j && jon) {
        const double fj = 4.0 * f;
        for (int sab = tid; sab < na * nb; sab += nt) {
            double s = 0.0;
            for (int t = 0; t < nscd; ++t) s += V[sab * nscd + t] * Pcd[t];
            atomicAdd(Jm + (long long)(a0 + sab / nb) * M + b0 + sab % nb, fj * s);
        }
        for (int scd = tid; scd < nscd; scd += nt) {
            double s = 0.0;
            for (int t = 0; t < na * nb; ++t) s += V[t * nscd + scd] * Pab[t];
            atomicAdd(Jm + (long long)(c0 + scd / nd) * M + d0 + scd % nd, fj * s);
        }
    }
    if (cl.want_k && kon) {
        const double fk = 2.0 * f;
        const int nac = na * nc, nad = na * nd, nbc = nb * nc, nbd = nb * nd;
        for (int e = tid; e < nac + nad + nbc + nbd; e += nt) {
            double s = 0.0;
            if (e < nac) {
                const int a = e / nc, c = e % nc;
                for (int b = 0; b < nb; ++b)
                    for (int d = 0; d < nd; ++d) s += V[(a * nb + b) * nscd + c * nd + d] * Pbd[b * nd + d];
                atomicAdd(Km + (long long)(a0 + a) * M + c0 + c, fk * s);
            } else if (e < nac + nad) {
                const int k = e - nac, a = k / nd, d = k % nd;
                for (int b = 0; b < nb; ++b)
                    for (int c = 0; c < nc; ++c) s += V[(a * nb + b) * nscd + c * nd + d] * Pbc[b * nc + c];
                atomicAdd(Km + (long long)(a0 + a) * M + d0 + d, fk * s);
            } else if (e < nac + nad + nbc) {
                const int k = e - nac - nad, b = k / nc, c = k % nc;
                for (int a = 0; a < na; ++a)
                    for (int d = 0; d < nd; ++d) s += V[(a * nb + b) * nscd + c * nd + d] * Pad[a * nd + d];
                atomicAdd(Km + (long long)(b0 + b) * M + c0 + c, fk * s);
            } else {
                const int k = e - nac - nad - nbc, b = k / nd, d = k % nd;
                for (int a = 0; a < na; ++a)
                    for (int c = 0; c < nc; ++c) s += V[(a * nb + b) * nscd + c * nd + d] * Pac[a * nc + c];
                atomicAdd(Km + (long long)(b0 + b) * M + d0 + d, fk * s);
            }
        }
    }
    __syncthreads();
}

// Tiled schedule (J/K mode), one quartet per block at a time: tile = 1 bra
// pair x bk ket pairs, tiles handed out by a block-wide dynamic counter.
template <typename R>
__global__ void eri_generic_cta_jk_kernel(PlanView pv, ClassLaunch cl, int nb_items) {
    extern __shared__ double smem[];
    GenericCtaLayout lay;
    lay.init(cl.la, cl.lb, cl.lc, cl.ld, nb_items);
    __shared__ int s_tile;
    const double thr = (cl.prec_mode != 0) ? cl.tau_mix / fmax(*cl.dmax, 1e-300) : 0.0;
    const int ntiles = cl.tile_end - cl.tile_begin;
    for (;;) {
        if (threadIdx.x == 0) s_tile = atomicAdd(cl.counter, 1);
        __syncthreads();
        const int t = s_tile;
        __syncthreads();
        if (t >= ntiles) break;
        const int tile = cl.tile_begin + t;
        const int b = find_block(cl.tile_prefix, cl.n_blocks, tile);
        const int kb = tile - __ldg(cl.tile_prefix + b);
        const BlockDesc bd = cl.blocks[b];
        const int bra = __ldg(cl.bra_list + bd.bra0);  // one bra per block
        const int i = bra - bd.xbeg;
        const double qi = pv.pair_Q[bra];
        for (int jj = 0; jj < cl.bk; ++jj) {
            const int j = kb * cl.bk + jj;
            if (j >= bd.nket) break;
            if (cl.same && bd.koff + j > i) break;
            const int ket = bd.ket0 + j;
            const double qq = qi * pv.pair_Q[ket];
            if (!(qq >= cl.tau)) continue;
            if (cl.prec_mode == 1 && !(qq >= thr)) continue;
            if (cl.prec_mode == 2 && qq >= thr) continue;
            bool lj = true, lk = true;
            if (cl.den.mode) {
                const int mol = pv.pair_mol ? pv.pair_mol[ket] : 0;
                density_live(cl, pv, mol, pv.pair_A[bra], pv.pair_B[bra], pv.pair_A[ket], pv.pair_B[ket], qq, lj, lk);
                if (!lj && !lk) continue;
            }
            generic_quartet_cta<R>(pv, cl, lay, smem, bra, ket, lj, lk);
        }
    }
}

}  // namespace dev
}  // namespace tlno_gpu
