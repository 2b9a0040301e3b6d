// Plan construction: shell pairs (oriented higher-L left, as the reference's
// pair groups, rys_engine.ipp:2449-2468), their primitive-pair records
// (rys_engine.ipp:2244-2279), exact Schwarz bounds Q_ab = max sqrt((ab|ab))
// computed on the device by the ERI kernel itself (the reference computes
// the same diagonal blocks, rys_engine.ipp:16165-16258), screening
// Q_ab Q_cd >= tau at shell-pair level (native_quartets.ipp:556-574), and the
// quartet-class schedules.
//
// Schedule: the pairs of every class are sorted by Q descending, so for a
// block of consecutive bra pairs the surviving kets of any class form a
// prefix of that class's list; a block's tile count is
// ceil(prefix / tile_kets).  The kernels map a linear tile id back to its
// block by binary search in the tile prefix sums and re-test every quartet.
#include "plan.hpp"

#include <algorithm>
#include <cmath>
#include <functional>
#include <numeric>
#include <thread>

#include "kernels.hpp"

namespace tlno_gpu {

namespace {
// Simint's binary64 FASTSCHWARZ prefactor sqrt(2) pi^{5/2} (the literal the
// reference keeps, rys_engine.ipp:68-72).
constexpr double kFastSchwarzPrefactor = 24.739429451193148050228357586821944304008810699990039583;

// Schwarz bucket of a pair: floor(-log2 Q), so bucket k holds
// Q in (2^-(k+1), 2^-k]; larger Q first.
int Q_bucket(double q) {
    if (!(q > 0.0)) return 1 << 20;
    int e = 0;
    const double m = std::frexp(q, &e);  // q = m 2^e, m in [0.5, 1)
    return (m == 0.5) ? 1 - e : -e;      // q == 2^(e-1) belongs to bucket 1-e
}
}  // namespace

namespace {

template <class T>
void upload_vec(DeviceBuffer& buf, const std::vector<T>& v, cudaStream_t s) {
    buf.alloc(std::max<std::size_t>(v.size() * sizeof(T), 16));
    if (!v.empty())
        TLNO_CUDA(cudaMemcpyAsync(buf.ptr, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s));
}

void parallel_for(long long n, const std::function<void(long long, long long)>& f) {
    const int nt = static_cast<int>(std::max(1u, std::min(16u, std::thread::hardware_concurrency())));
    if (n < 4096 || nt == 1) {
        f(0, n);
        return;
    }
    std::vector<std::thread> ts;
    const long long chunk = (n + nt - 1) / nt;
    for (int t = 0; t < nt; ++t) {
        const long long b = t * chunk, e = std::min(n, b + chunk);
        if (b >= e) break;
        ts.emplace_back(f, b, e);
    }
    for (auto& t : ts) t.join();
}

inline void oriented(const Basis& b, int i, int j, int& A, int& B) {
    A = i;
    B = j;
    if (b.shells[B].L > b.shells[A].L) std::swap(A, B);
}

// Algorithmic flop model per primitive quartet (native-route operation
// count): 30 + N [40 + 15 + 3 V_axis + 3 nc(a)nc(b)nc(c)nc(d)],
// V_axis = 5(LAB+1)(LCD+1) + 2 sum_{j=1..b}(LAB-j+1)(LCD+1)
//        + 2 sum_{l=1..d}(a+1)(b+1)(LCD-l+1).
double flops_per_prim(int a, int b, int c, int d) {
    const int LAB = a + b, LCD = c + d, N = (LAB + LCD) / 2 + 1;
    double vaxis = 5.0 * (LAB + 1) * (LCD + 1);
    for (int j = 1; j <= b; ++j) vaxis += 2.0 * (LAB - j + 1) * (LCD + 1);
    for (int l = 1; l <= d; ++l) vaxis += 2.0 * (a + 1) * (b + 1) * (LCD - l + 1);
    const double ncart4 = double(n_cart(a)) * n_cart(b) * n_cart(c) * n_cart(d);
    return 30.0 + N * (40.0 + 15.0 + 3.0 * vaxis + 3.0 * ncart4);
}
// Per contracted quartet: 2 x projection terms + 12 per spherical ERI.
double flops_per_contracted(int a, int b, int c, int d) {
    const double ncart4 = double(n_cart(a)) * n_cart(b) * n_cart(c) * n_cart(d);
    const double nsph4 = double(n_sph(a)) * n_sph(b) * n_sph(c) * n_sph(d);
    return 2.0 * 2.0 * ncart4 + 12.0 * nsph4;
}

}  // namespace

int primitive_pair_count(const Basis& b, int A, int B) {
    const Shell& sa = b.shells[A];
    const Shell& sb = b.shells[B];
    int n = 0;
    for (int i = 0; i < sa.nprim; ++i)
        for (int j = 0; j < sb.nprim; ++j)
            if (b.c_radial[sa.prim_offset + i] * b.c_radial[sb.prim_offset + j] != 0.0) ++n;
    return n;
}

void primitive_pairs(const Basis& b, int A, int B, std::vector<dev::DPrimPair>& out) {
    const Shell& sa = b.shells[A];
    const Shell& sb = b.shells[B];
    const double* a = sa.center;
    const double* c = sb.center;
    const double ab[3] = {a[0] - c[0], a[1] - c[1], a[2] - c[2]};
    const double r2 = ab[0] * ab[0] + ab[1] * ab[1] + ab[2] * ab[2];
    for (int i = 0; i < sa.nprim; ++i) {
        const double al = b.exps[sa.prim_offset + i];
        const double ca = b.c_radial[sa.prim_offset + i];
        for (int j = 0; j < sb.nprim; ++j) {
            const double be = b.exps[sb.prim_offset + j];
            const double cab = ca * b.c_radial[sb.prim_offset + j];
            if (cab == 0.0) continue;
            const double p = al + be, invp = 1.0 / p;
            const double K = std::exp(-(al * be * invp) * r2);
            dev::DPrimPair pp;
            pp.p = p;
            pp.invp = invp;
            pp.Px = (al * a[0] + be * c[0]) * invp;
            pp.Py = (al * a[1] + be * c[1]) * invp;
            pp.Pz = (al * a[2] + be * c[2]) * invp;
            pp.w = K * cab * invp;
            out.push_back(pp);
        }
    }
}

// Decay scale of a shell (alpha_min, K = sum_i |c_i| (pi / alpha_i)^{3/4})
// and the pair indicator K_A K_B exp(-mu |AB|^2), mu from the two smallest
// exponents (rys_engine.ipp:2205-2241).
namespace {
struct DecayScale {
    double alpha_min = 0.0, K = 0.0;
};
DecayScale decay_scale(const Basis& b, int sh) {
    const Shell& s = b.shells[sh];
    DecayScale out;
    if (s.nprim == 0) return out;
    out.alpha_min = b.exps[s.prim_offset];
    for (int i = 0; i < s.nprim; ++i) {
        const double alpha = b.exps[s.prim_offset + i];
        out.alpha_min = std::min(out.alpha_min, alpha);
        out.K += std::fabs(b.c_radial[s.prim_offset + i]) * std::pow(kPi / alpha, 0.75);
    }
    return out;
}
double pair_decay_bound(const Basis& b, int A, int B, const DecayScale& a, const DecayScale& c) {
    if (!(a.alpha_min > 0.0) || !(c.alpha_min > 0.0)) return 0.0;
    const double dx = b.shells[A].center[0] - b.shells[B].center[0];
    const double dy = b.shells[A].center[1] - b.shells[B].center[1];
    const double dz = b.shells[A].center[2] - b.shells[B].center[2];
    const double r2 = dx * dx + dy * dy + dz * dz;
    const double mu = a.alpha_min * c.alpha_min / (a.alpha_min + c.alpha_min);
    return a.K * c.K * std::exp(-mu * r2);
}
}  // namespace

MolPairs build_mol_pairs(const Basis& b, double tau, cudaStream_t s, double decay) {
    MolPairs mp;
    const int ns = static_cast<int>(b.shells.size());
    const long long npairs = static_cast<long long>(ns) * (ns + 1) / 2;
    mp.Q_canonical.assign(static_cast<std::size_t>(npairs), 0.0);
    if (ns == 0) return mp;
    const bool use_decay = decay > 0.0;
    if (use_decay) tau = decay;
    std::vector<DecayScale> dscale;
    if (use_decay)
        for (int i = 0; i < ns; ++i) dscale.push_back(decay_scale(b, i));

    // Device copy of the shells for the Schwarz kernel.
    std::vector<double> xyz(3 * ns);
    std::vector<int> Ls(ns), sph(ns);
    for (int i = 0; i < ns; ++i) {
        for (int k = 0; k < 3; ++k) xyz[3 * i + k] = b.shells[i].center[k];
        Ls[i] = b.shells[i].L;
        sph[i] = b.shells[i].sph_offset;
    }
    DeviceBuffer d_xyz, d_L, d_sph;
    upload_vec(d_xyz, xyz, s);
    upload_vec(d_L, Ls, s);
    upload_vec(d_sph, sph, s);

    // Chunked evaluation of the diagonal quartets (ab|ab).
    const long long chunk = 1 << 20;
    DeviceBuffer d_A, d_B, d_off, d_np, d_prim, d_list, d_Q;
    for (long long c0 = 0; c0 < npairs; c0 += chunk) {
        const long long c1 = std::min(npairs, c0 + chunk);
        const int n = static_cast<int>(c1 - c0);
        std::vector<int> A(n), B(n), np(n), off(n + 1, 0), cls(n);
        // canonical pair index t -> (i, j), i >= j
        long long i = static_cast<long long>((std::sqrt(8.0 * c0 + 1.0) - 1.0) / 2.0);
        while (i * (i + 1) / 2 > c0) --i;
        while ((i + 1) * (i + 2) / 2 <= c0) ++i;
        long long j = c0 - i * (i + 1) / 2;
        for (int t = 0; t < n; ++t) {
            int a, bb;
            oriented(b, static_cast<int>(i), static_cast<int>(j), a, bb);
            A[t] = a;
            B[t] = bb;
            np[t] = primitive_pair_count(b, a, bb);
            cls[t] = pair_class_of(b.shells[a].L, b.shells[bb].L);
            if (++j > i) { ++i; j = 0; }
        }
        for (int t = 0; t < n; ++t) off[t + 1] = off[t] + np[t];
        std::vector<dev::DPrimPair> prim(static_cast<std::size_t>(off[n]));
        parallel_for(n, [&](long long b0, long long e0) {
            std::vector<dev::DPrimPair> tmp;
            for (long long t = b0; t < e0; ++t) {
                tmp.clear();
                primitive_pairs(b, A[t], B[t], tmp);
                std::copy(tmp.begin(), tmp.end(), prim.begin() + off[t]);
            }
        });
        upload_vec(d_A, A, s);
        upload_vec(d_B, B, s);
        upload_vec(d_off, off, s);
        upload_vec(d_np, np, s);
        upload_vec(d_prim, prim, s);
        d_Q.alloc(sizeof(double) * n);
        dev::PlanView pv{};
        pv.shell_xyz = d_xyz.as<double>();
        pv.shell_L = d_L.as<int>();
        pv.shell_sph = d_sph.as<int>();
        pv.pair_A = d_A.as<int>();
        pv.pair_B = d_B.as<int>();
        pv.pair_prim_off = d_off.as<int>();
        pv.pair_nprim = d_np.as<int>();
        pv.prim = d_prim.as<dev::DPrimPair>();
        // one launch per pair class
        std::vector<std::vector<int>> by_cls(kMaxPairClasses);
        for (int t = 0; t < n; ++t) by_cls[cls[t]].push_back(t);
        std::vector<int> list;
        std::vector<int> list_off(kMaxPairClasses + 1, 0);
        for (int c = 0; c < kMaxPairClasses; ++c) {
            list_off[c + 1] = list_off[c] + static_cast<int>(by_cls[c].size());
            list.insert(list.end(), by_cls[c].begin(), by_cls[c].end());
        }
        upload_vec(d_list, list, s);
        for (int c = 0; c < kMaxPairClasses && !use_decay; ++c) {
            const int cnt = list_off[c + 1] - list_off[c];
            if (cnt == 0) continue;
            int la = 0;
            while ((la + 1) * (la + 2) / 2 <= c) ++la;
            const int lb = c - la * (la + 1) / 2;
            dev::ClassLaunch cl{};
            cl.la = la; cl.lb = lb; cl.lc = la; cl.ld = lb;
            cl.q_bra = d_list.as<int>() + list_off[c];
            cl.q_ket = cl.q_bra;
            cl.n_quartets = cnt;
            cl.out = d_Q.as<double>() + list_off[c];
            launch_eri_schwarz(pv, cl, s);
        }
        if (use_decay) {
            for (int t = 0; t < n; ++t) mp.Q_canonical[c0 + t] = pair_decay_bound(b, A[t], B[t], dscale[A[t]], dscale[B[t]]);
        } else {
            std::vector<double> qsorted(n);
            TLNO_CUDA(cudaMemcpyAsync(qsorted.data(), d_Q.ptr, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
            TLNO_CUDA(cudaStreamSynchronize(s));
            for (int pos = 0; pos < n; ++pos) mp.Q_canonical[c0 + list[pos]] = qsorted[pos];
        }
        // remember pair metadata in canonical order for the selection below
        for (int t = 0; t < n; ++t) {
            mp.A.push_back(A[t]);
            mp.B.push_back(B[t]);
            mp.nprim.push_back(np[t]);
            mp.cls.push_back(cls[t]);
        }
    }
    for (double q : mp.Q_canonical) mp.Qmax = std::max(mp.Qmax, q);
    // Keep pairs that can pass Q_ab * Q_cd >= tau for some cd; sort by
    // class then Q descending (ties by canonical index).
    std::vector<long long> keep;
    keep.reserve(static_cast<std::size_t>(npairs));
    for (long long t = 0; t < npairs; ++t) {
        if (tau > 0.0 && !(mp.Q_canonical[t] * mp.Qmax >= tau)) continue;
        keep.push_back(t);
    }
    // Inside a class, pairs are grouped by primitive count (a tile of kets
    // then runs one primitive loop length on every lane), then by Schwarz
    // bucket floor(-log2 Q) (the kets that can pass the bound for a bra form
    // a prefix of whole buckets), and inside a bucket by shell indices, so
    // that neighbouring lanes read and update neighbouring density and J/K
    // elements.
    auto bucket = [&](long long t) { return Q_bucket(mp.Q_canonical[t]); };
    std::stable_sort(keep.begin(), keep.end(), [&](long long l, long long r) {
        if (mp.cls[l] != mp.cls[r]) return mp.cls[l] < mp.cls[r];
        if (mp.nprim[l] != mp.nprim[r]) return mp.nprim[l] < mp.nprim[r];
        const int bl = bucket(l), br = bucket(r);
        if (bl != br) return bl < br;
        if (mp.A[l] != mp.A[r]) return mp.A[l] < mp.A[r];
        return mp.B[l] < mp.B[r];
    });
    MolPairs out;
    out.Q_canonical = std::move(mp.Q_canonical);
    out.Qmax = mp.Qmax;
    out.cls_begin.fill(0);
    out.cls_count.fill(0);
    for (std::size_t k = 0; k < keep.size(); ++k) {
        const long long t = keep[k];
        out.A.push_back(mp.A[t]);
        out.B.push_back(mp.B[t]);
        out.nprim.push_back(mp.nprim[t]);
        out.cls.push_back(mp.cls[t]);
        out.Q.push_back(out.Q_canonical[t]);
        out.cls_count[mp.cls[t]]++;
    }
    int acc = 0;
    for (int c = 0; c < kMaxPairClasses; ++c) {
        out.cls_begin[c] = acc;
        acc += out.cls_count[c];
    }
    return out;
}

dev::PlanView Plan2e::view() const {
    dev::PlanView pv{};
    pv.shell_xyz = d_shell_xyz.as<double>();
    pv.shell_L = d_shell_L.as<int>();
    pv.shell_sph = d_shell_sph.as<int>();
    pv.pair_A = d_pair_A.as<int>();
    pv.pair_B = d_pair_B.as<int>();
    pv.pair_prim_off = d_pair_prim_off.as<int>();
    pv.pair_nprim = d_pair_nprim.as<int>();
    pv.pair_Q = d_pair_Q.as<double>();
    pv.pair_mol = n_mol > 1 ? d_pair_mol.as<int>() : nullptr;
    pv.prim = d_prim.as<dev::DPrimPair>();
    pv.prim32 = d_prim32.as<dev::FPrimPair>();
    pv.mol_mat_off = n_mol > 1 ? d_mol_mat_off.as<long long>() : nullptr;
    pv.mol_M = n_mol > 1 ? d_mol_M.as<int>() : nullptr;
    pv.prim_fs = d_prim_fs.as<double>();
    pv.mol_shell_off = n_mol > 1 ? d_mol_shell_off.as<int>() : nullptr;
    pv.mol_ns = n_mol > 1 ? d_mol_ns.as<int>() : nullptr;
    pv.proj = proj_ready ? d_proj.as<double>() : nullptr;
    pv.proj_off = proj_ready ? d_proj_off.as<long long>() : nullptr;
    return pv;
}

void build_plan(Plan2e& plan, const std::vector<const Basis*>& bases, std::vector<MolPairs>&& pairs,
                double tau, const Tuning& tune, cudaStream_t s) {
    plan.tau = tau;
    plan.n_mol = static_cast<int>(bases.size());
    plan.mol_pairs = std::move(pairs);
    plan.mol_shell_off.assign(plan.n_mol + 1, 0);
    plan.mol_M.assign(plan.n_mol, 0);
    plan.mol_mat_off.assign(plan.n_mol + 1, 0);
    std::vector<double> xyz;
    std::vector<int> Ls, sph;
    for (int m = 0; m < plan.n_mol; ++m) {
        const Basis& b = *bases[m];
        plan.mol_shell_off[m + 1] = plan.mol_shell_off[m] + static_cast<int>(b.shells.size());
        plan.mol_M[m] = b.n_sph;
        plan.mol_mat_off[m + 1] = plan.mol_mat_off[m] + static_cast<long long>(b.n_sph) * b.n_sph;
        for (const Shell& sh : b.shells) {
            xyz.insert(xyz.end(), sh.center, sh.center + 3);
            Ls.push_back(sh.L);
            sph.push_back(sh.sph_offset);
        }
    }
    // Global sorted pair arrays: per molecule the class-sorted list; the
    // class lists of one molecule are contiguous.
    std::vector<std::array<int, kMaxPairClasses>> gbeg(plan.n_mol);
    plan.pair_A.clear(); plan.pair_B.clear(); plan.pair_nprim.clear();
    plan.pair_prim_off.clear(); plan.pair_Q.clear(); plan.pair_mol.clear();
    plan.total_pairs = 0;
    int prim_total = 0;
    for (int m = 0; m < plan.n_mol; ++m) {
        const MolPairs& mp = plan.mol_pairs[m];
        const int base = static_cast<int>(plan.pair_A.size());
        for (int c = 0; c < kMaxPairClasses; ++c) gbeg[m][c] = base + mp.cls_begin[c];
        const int so = plan.mol_shell_off[m];
        for (std::size_t k = 0; k < mp.A.size(); ++k) {
            plan.pair_A.push_back(mp.A[k] + so);
            plan.pair_B.push_back(mp.B[k] + so);
            plan.pair_nprim.push_back(mp.nprim[k]);
            plan.pair_prim_off.push_back(prim_total);
            prim_total += mp.nprim[k];
            plan.pair_Q.push_back(mp.Q[k]);
            plan.pair_mol.push_back(m);
        }
        const long long ns = bases[m]->shells.size();
        plan.total_pairs += ns * (ns + 1) / 2;
    }
    plan.kept_pairs = static_cast<long long>(plan.pair_A.size());
    std::vector<dev::DPrimPair> prim(static_cast<std::size_t>(prim_total));
    std::vector<dev::FPrimPair> prim32(static_cast<std::size_t>(prim_total));
    std::vector<double> prim_fs(static_cast<std::size_t>(prim_total));
    {
        const long long np = static_cast<long long>(plan.pair_A.size());
        parallel_for(np, [&](long long b0, long long e0) {
            std::vector<dev::DPrimPair> tmp;
            for (long long k = b0; k < e0; ++k) {
                const int m = plan.pair_mol[k];
                const int so = plan.mol_shell_off[m];
                tmp.clear();
                primitive_pairs(*bases[m], plan.pair_A[k] - so, plan.pair_B[k] - so, tmp);
                std::copy(tmp.begin(), tmp.end(), prim.begin() + plan.pair_prim_off[k]);
                const auto& ca = bases[m]->shells[plan.pair_A[k] - so].center;
                for (std::size_t t = 0; t < tmp.size(); ++t) {
                    const dev::DPrimPair& d = tmp[t];
                    // Simint's FASTSCHWARZ primitive-pair value, squared MEST
                    // estimate sqrt(2) pi^{5/2} p^{-5/2} e^{-2 mu R^2} (cA cB)^2
                    // (rys_engine.ipp:68-72, 2264-2268)
                    prim_fs[plan.pair_prim_off[k] + t] = kFastSchwarzPrefactor * d.w * d.w * std::sqrt(d.invp);
                    prim32[plan.pair_prim_off[k] + t] = {static_cast<float>(d.p), static_cast<float>(d.Px - ca[0]),
                                                         static_cast<float>(d.Py - ca[1]), static_cast<float>(d.Pz - ca[2]),
                                                         static_cast<float>(d.w), static_cast<float>(d.invp)};
                }
            }
        });
    }
    upload_vec(plan.d_shell_xyz, xyz, s);
    upload_vec(plan.d_shell_L, Ls, s);
    upload_vec(plan.d_shell_sph, sph, s);
    upload_vec(plan.d_pair_A, plan.pair_A, s);
    upload_vec(plan.d_pair_B, plan.pair_B, s);
    upload_vec(plan.d_pair_nprim, plan.pair_nprim, s);
    upload_vec(plan.d_pair_prim_off, plan.pair_prim_off, s);
    upload_vec(plan.d_pair_Q, plan.pair_Q, s);
    upload_vec(plan.d_pair_mol, plan.pair_mol, s);
    upload_vec(plan.d_prim, prim, s);
    upload_vec(plan.d_prim32, prim32, s);
    upload_vec(plan.d_mol_mat_off, plan.mol_mat_off, s);
    upload_vec(plan.d_mol_M, plan.mol_M, s);
    upload_vec(plan.d_prim_fs, prim_fs, s);
    plan.mol_ns.assign(plan.n_mol, 0);
    plan.rho_off.assign(plan.n_mol + 1, 0);
    plan.max_ns2 = 0;
    for (int m = 0; m < plan.n_mol; ++m) {
        plan.mol_ns[m] = plan.mol_shell_off[m + 1] - plan.mol_shell_off[m];
        const long long n2 = static_cast<long long>(plan.mol_ns[m]) * plan.mol_ns[m];
        plan.rho_off[m + 1] = plan.rho_off[m] + n2;
        plan.max_ns2 = std::max(plan.max_ns2, n2);
    }
    upload_vec(plan.d_mol_shell_off, plan.mol_shell_off, s);
    upload_vec(plan.d_mol_ns, plan.mol_ns, s);
    upload_vec(plan.d_rho_off, plan.rho_off, s);

    // Quartet-class schedules.
    plan.combos.clear();
    plan.total_quartets = plan.total_prim_quartets = 0;
    plan.total_flops = 0.0;
    for (int X = 0; X < kMaxPairClasses; ++X) {
        for (int Y = 0; Y <= X; ++Y) {
            ComboSchedule cs;
            cs.X = X;
            cs.Y = Y;
            int la = 0;
            while ((la + 1) * (la + 2) / 2 <= X) ++la;
            int lc = 0;
            while ((lc + 1) * (lc + 2) / 2 <= Y) ++lc;
            cs.la = la; cs.lb = X - la * (la + 1) / 2;
            cs.lc = lc; cs.ld = Y - lc * (lc + 1) / 2;
            const int combo_id = X * kMaxPairClasses + Y;
            cs.fast = has_fast_kernel(cs.la, cs.lb, cs.lc, cs.ld) &&
                      !(combo_id < 256 && tune.force_generic[combo_id]);
            cs.bb = cs.fast ? fast_kernel_bras(cs.la, cs.lb, cs.lc, cs.ld) : 1;
            cs.bk = cs.fast ? 32 : tune.generic_bk;
            const double fprim = flops_per_prim(cs.la, cs.lb, cs.lc, cs.ld);
            const double fcon = flops_per_contracted(cs.la, cs.lb, cs.lc, cs.ld);
            cs.prefix.push_back(0);
            for (int m = 0; m < plan.n_mol; ++m) {
                const MolPairs& mp = plan.mol_pairs[m];
                const int nX = mp.cls_count[X], nY = mp.cls_count[Y];
                if (nX == 0 || nY == 0) continue;
                const int bx0 = gbeg[m][X], by0 = gbeg[m][Y];
                // ket segments of equal primitive count
                std::vector<int> seg{0};
                for (int j = 1; j < nY; ++j)
                    if (plan.pair_nprim[by0 + j] != plan.pair_nprim[by0 + j - 1]) seg.push_back(j);
                seg.push_back(nY);
                const double* qk = plan.pair_Q.data() + by0;
                // Per segment: Q sorted descending (exact quartet counts) and,
                // per position, the largest Q of its bucket (non-increasing
                // along the segment) for the schedule extent.
                std::vector<double> qsorted(qk, qk + nY), bmax(nY);
                for (std::size_t sg = 0; sg + 1 < seg.size(); ++sg) {
                    const int s0 = seg[sg], s1 = seg[sg + 1];
                    std::sort(qsorted.begin() + s0, qsorted.begin() + s1, std::greater<double>());
                    for (int j = s0; j < s1;) {
                        int e = j;
                        double mx = 0.0;
                        const int bk = Q_bucket(qk[j]);
                        while (e < s1 && Q_bucket(qk[e]) == bk) mx = std::max(mx, qk[e++]);
                        for (int t = j; t < e; ++t) bmax[t] = mx;
                        j = e;
                    }
                }
                // Tile extent of segment [s0, s1) for a bra of bound qi: the
                // whole buckets that may hold a passing ket (on the diagonal
                // class only local index <= i).
                auto seg_extent = [&](double qi, int s0, int s1, int i) {
                    int lo = s1;
                    if (tau > 0.0) {
                        lo = s0;
                        int hi = s1;
                        while (lo < hi) {
                            const int mid = (lo + hi) / 2;
                            if (qi * bmax[mid] >= tau) lo = mid + 1; else hi = mid;
                        }
                    }
                    int e = lo - s0;
                    if (X == Y) e = std::min(e, i + 1 - s0);
                    return std::max(e, 0);
                };
                // passing kets of segment [s0, s1) for a bra of bound qi
                auto seg_count = [&](double qi, int s0, int s1) {
                    if (tau <= 0.0) return s1 - s0;
                    int a = s0, b = s1;
                    while (a < b) {
                        const int mid = (a + b) / 2;
                        if (qi * qsorted[mid] >= tau) a = mid + 1; else b = mid;
                    }
                    return a - s0;
                };
                // Exact surviving quartets and primitive quartets.  Off the
                // diagonal every (bra, ket) pair counts; on the diagonal class
                // (one list, j <= i) a ket segment before the bra's segment
                // counts fully and the bra's own segment holds
                // (ordered pairs + self pairs) / 2.
                {
                    std::vector<int> seg_of(nX);
                    if (X == Y)
                        for (std::size_t sg = 0; sg + 1 < seg.size(); ++sg)
                            for (int j = seg[sg]; j < seg[sg + 1]; ++j) seg_of[j] = static_cast<int>(sg);
                    std::vector<long long> own_ordered(seg.size(), 0), own_self(seg.size(), 0);
                    for (int i = 0; i < nX; ++i) {
                        const double qi = plan.pair_Q[bx0 + i];
                        const long long npb = plan.pair_nprim[bx0 + i];
                        for (std::size_t sg = 0; sg + 1 < seg.size(); ++sg) {
                            if (X == Y && static_cast<int>(sg) > seg_of[i]) break;
                            const int c = seg_count(qi, seg[sg], seg[sg + 1]);
                            if (X == Y && static_cast<int>(sg) == seg_of[i]) {
                                own_ordered[sg] += c;
                                if (tau <= 0.0 || qi * qi >= tau) own_self[sg] += 1;
                                continue;
                            }
                            cs.quartets += c;
                            cs.prim_quartets += npb * plan.pair_nprim[by0 + seg[sg]] * c;
                        }
                    }
                    if (X == Y)
                        for (std::size_t sg = 0; sg + 1 < seg.size(); ++sg) {
                            const long long n = (own_ordered[sg] + own_self[sg]) / 2;
                            const long long np = plan.pair_nprim[by0 + seg[sg]];
                            cs.quartets += n;
                            cs.prim_quartets += np * np * n;
                        }
                }
                // Bra order: the class list order, or (bra groups) grouped by
                // first shell A inside each primitive-count group, list order
                // kept inside a group; a block holds up to cs.bb bras of one A.
                std::vector<int> order(nX);
                for (int i = 0; i < nX; ++i) order[i] = i;
                if (cs.bb > 1)
                    std::stable_sort(order.begin(), order.end(), [&](int u, int v) {
                        const int nu = plan.pair_nprim[bx0 + u], nv = plan.pair_nprim[bx0 + v];
                        if (nu != nv) return nu < nv;
                        return plan.pair_A[bx0 + u] < plan.pair_A[bx0 + v];
                    });
                for (int i0 = 0; i0 < nX;) {
                    int nbra = 1;
                    if (cs.bb > 1)
                        while (nbra < cs.bb && i0 + nbra < nX &&
                               plan.pair_A[bx0 + order[i0 + nbra]] == plan.pair_A[bx0 + order[i0]])
                            ++nbra;
                    const int brabeg = static_cast<int>(cs.bra_list.size());
                    bool used = false;
                    for (std::size_t sg = 0; sg + 1 < seg.size(); ++sg) {
                        const int s0 = seg[sg], s1 = seg[sg + 1];
                        int ext = 0;
                        for (int w = 0; w < nbra; ++w) {
                            const int i = order[i0 + w];
                            ext = std::max(ext, seg_extent(plan.pair_Q[bx0 + i], s0, s1, i));
                        }
                        const int nt = (ext + cs.bk - 1) / cs.bk;
                        if (nt <= 0) continue;
                        used = true;
                        dev::BlockDesc bd{};
                        bd.bra0 = brabeg;
                        bd.nbra = nbra;
                        bd.ket0 = by0 + s0;
                        bd.nket = s1 - s0;
                        bd.xbeg = bx0;
                        bd.koff = s0;
                        cs.blocks.push_back(bd);
                        cs.prefix.push_back(cs.prefix.back() + nt);
                    }
                    if (used)
                        for (int w = 0; w < nbra; ++w) cs.bra_list.push_back(bx0 + order[i0 + w]);
                    i0 += nbra;
                }
            }
            cs.n_tiles = cs.prefix.back();
            if (cs.n_tiles == 0) continue;
            cs.flops = fprim * cs.prim_quartets + fcon * cs.quartets;
            upload_vec(cs.d_blocks, cs.blocks, s);
            upload_vec(cs.d_prefix, cs.prefix, s);
            upload_vec(cs.d_bra_list, cs.bra_list, s);
            plan.total_quartets += cs.quartets;
            plan.total_prim_quartets += cs.prim_quartets;
            plan.total_flops += cs.flops;
            plan.combos.push_back(std::move(cs));
        }
    }
    plan.d_counters.alloc(sizeof(int) * 2 * std::max<std::size_t>(plan.combos.size(), 1));

    // HRR + spherical projectors of the pairs of every pair class that a
    // generic (CTA) class combination uses, built once on the device.
    {
        std::array<bool, kMaxPairClasses> need{};
        for (const ComboSchedule& cs : plan.combos)
            if (!cs.fast) need[cs.X] = need[cs.Y] = true;
        const std::size_t np = plan.pair_A.size();
        plan.proj_off.assign(np, -1);
        long long words = 0;
        for (std::size_t k = 0; k < np; ++k) {
            const int la = Ls[plan.pair_A[k]], lb = Ls[plan.pair_B[k]];
            if (!need[la * (la + 1) / 2 + lb]) continue;
            plan.proj_off[k] = words;
            const int nslice = (la + lb + 1) * (la + lb + 2) * (la + lb + 3) / 6 - la * (la + 1) * (la + 2) / 6;
            words += static_cast<long long>(2 * la + 1) * (2 * lb + 1) * nslice;
        }
        plan.proj_words = words;
        plan.proj_ready = false;
        if (words > 0 && words * 8 <= kMaxProjectorBytes) {
            plan.d_proj.alloc(sizeof(double) * words);
            upload_vec(plan.d_proj_off, plan.proj_off, s);
            launch_pair_projectors(plan.d_pair_A.as<int>(), plan.d_pair_B.as<int>(), plan.d_shell_xyz.as<double>(),
                                   plan.d_shell_L.as<int>(), plan.d_proj_off.as<long long>(), static_cast<int>(np),
                                   plan.d_proj.as<double>(), s);
            plan.proj_ready = true;
        }
    }
    TLNO_CUDA(cudaStreamSynchronize(s));
}

void ensure_density_tables(Plan2e& plan) {
    plan.d_rho_blk.alloc(sizeof(double) * std::max<long long>(plan.rho_off.empty() ? 1 : plan.rho_off.back(), 1));
    plan.d_rho_max.alloc(sizeof(double) * std::max(plan.n_mol, 1));
}

void build_onee_plan(OneePlan& p, const Basis& b, double decay_eps, double nuclear_eps) {
    const int ns = static_cast<int>(b.shells.size());
    p.pairs.clear();
    // Group decay scales from the representative shell of each group:
    // alpha_min and K = sum_i |c_i| (pi / alpha_i)^{3/4} with the normalised
    // coefficient of the group's first Cartesian component (x^L).
    const int ng = static_cast<int>(b.onee_group_rep.size());
    std::vector<double> amin(ng, 1e300), Kd(ng, 0.0);
    auto c_first = [&](const Shell& s, int i) {
        double df = 1.0;
        for (int k = 2 * s.L - 1; k > 0; k -= 2) df *= k;
        return b.c_radial[s.prim_offset + i] / std::sqrt(df);
    };
    for (int g = 0; g < ng; ++g) {
        const Shell& s = b.shells[b.onee_group_rep[g]];
        for (int i = 0; i < s.nprim; ++i) {
            const double a = b.exps[s.prim_offset + i];
            amin[g] = std::min(amin[g], a);
            Kd[g] += std::fabs(c_first(s, i)) * std::pow(kPi / a, 0.75);
        }
    }
    // Per-primitive max |normalised coefficient| over the group's components.
    p.maxc.assign(b.exps.size(), 0.0);
    std::vector<std::vector<double>> gmax(ng);
    for (int si = 0; si < ns; ++si) {
        const Shell& s = b.shells[si];
        const int g = b.onee_group[si];
        gmax[g].resize(s.nprim, 0.0);
        double maxang = 0.0;
        for (int x = s.L; x >= 0; --x)
            for (int y = s.L - x; y >= 0; --y) {
                const int z = s.L - x - y;
                double df = 1.0;
                for (int k = 2 * x - 1; k > 0; k -= 2) df *= k;
                for (int k = 2 * y - 1; k > 0; k -= 2) df *= k;
                for (int k = 2 * z - 1; k > 0; k -= 2) df *= k;
                maxang = std::max(maxang, 1.0 / std::sqrt(df));
            }
        for (int i = 0; i < s.nprim; ++i)
            gmax[g][i] = std::max(gmax[g][i], std::fabs(b.c_radial[s.prim_offset + i]) * maxang);
    }
    for (int si = 0; si < ns; ++si) {
        const Shell& s = b.shells[si];
        for (int i = 0; i < s.nprim; ++i) p.maxc[s.prim_offset + i] = gmax[b.onee_group[si]][i];
    }
    for (int i = 0; i < ns; ++i) {
        for (int j = 0; j <= i; ++j) {
            const int gi = b.onee_group[i], gj = b.onee_group[j];
            const Shell& si_ = b.shells[i];
            const Shell& sj_ = b.shells[j];
            const double dx = si_.center[0] - sj_.center[0], dy = si_.center[1] - sj_.center[1],
                         dz = si_.center[2] - sj_.center[2];
            const double r2 = dx * dx + dy * dy + dz * dz;
            bool keep = true;
            double bound = 0.0;
            if (decay_eps > 0.0) {
                const double mu = amin[gi] * amin[gj] / (amin[gi] + amin[gj]);
                if (Kd[gi] * Kd[gj] * std::exp(-mu * r2) < decay_eps) keep = false;
                if (keep) {
                    const Shell& ri = b.shells[b.onee_group_rep[gi]];
                    const Shell& rj = b.shells[b.onee_group_rep[gj]];
                    for (int a = 0; a < ri.nprim; ++a)
                        for (int c = 0; c < rj.nprim; ++c) {
                            const double ea = b.exps[ri.prim_offset + a], ec = b.exps[rj.prim_offset + c];
                            const double pp = ea + ec, chi = ea * ec / pp;
                            bound += std::fabs(c_first(ri, a) * c_first(rj, c)) * std::pow(kPi / pp, 1.5) *
                                     std::exp(-chi * r2);
                        }
                }
            }
            if (!keep) continue;
            dev::OneePair op{};
            op.A = i;
            op.B = j;
            if (b.shells[j].L > b.shells[i].L) std::swap(op.A, op.B);
            op.do_st = 1;
            op.do_v = (decay_eps <= 0.0 || bound >= decay_eps) ? 1 : 0;
            p.pairs.push_back(op);
        }
    }
    p.nuc.clear();
    double zsum = 0.0;
    for (std::size_t a = 0; a < b.Z.size(); ++a) {
        zsum += std::fabs(static_cast<double>(b.Z[a]));
        if (b.Z[a] == 0) continue;
        p.nuc.push_back(b.atom_xyz[3 * a]);
        p.nuc.push_back(b.atom_xyz[3 * a + 1]);
        p.nuc.push_back(b.atom_xyz[3 * a + 2]);
        p.nuc.push_back(static_cast<double>(b.Z[a]));
    }
    p.screen_thr = (zsum > 0.0) ? nuclear_eps / zsum : 0.0;
}

}  // namespace tlno_gpu
