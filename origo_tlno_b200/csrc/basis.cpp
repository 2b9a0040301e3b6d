// Basis construction and validation.
//
// Raw contracted shells are normalised exactly as the reference's make_shell
// does it (core/shell/shell_contract.cpp:9-48, shell_math.cpp:50-77): each
// primitive gets sqrt(2^(2L+1.5) a^(L+1.5) / (pi^1.5 prod (2l-1)!!)) and the
// contraction is rescaled to unit self-overlap.  The engine keeps the radial
// coefficient c_radial = c(L,0,0) / N_ang(L,0,0) per primitive, which every
// Cartesian component shares (rys_engine.ipp:2044-2058).
// Validation follows the reference's error contract: finite centres and
// coefficients, positive finite exponents, at least one primitive, L in 0..4
// (rys_engine.ipp:1967-2000, 2374-2383).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "engine.hpp"

namespace tlno_gpu {

void cuda_check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        throw Error(-2, std::string("CUDA error: ") + cudaGetErrorString(e) + " in " + what);
    }
}

void DeviceBuffer::release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
}

void DeviceBuffer::alloc(std::size_t n) {
    if (n <= bytes && ptr) return;
    release();
    if (n == 0) return;
    TLNO_CUDA(cudaMalloc(&ptr, n));
    bytes = n;
}

namespace {

inline bool finite_bits(double v) {
    std::uint64_t bits;
    std::memcpy(&bits, &v, sizeof(bits));
    return (bits & 0x7ff0000000000000ull) != 0x7ff0000000000000ull;
}

double double_factorial(int n) {
    double r = 1.0;
    for (int k = n; k > 0; k -= 2) r *= k;
    return r;
}

double ang_norm(int lx, int ly, int lz) {
    return 1.0 / std::sqrt(double_factorial(2 * lx - 1) * double_factorial(2 * ly - 1) *
                           double_factorial(2 * lz - 1));
}

// Normalised coefficients of the (L, 0, 0) component (make_shell).
std::vector<double> normalise_xl(int L, const double* exps, const double* coefs, int nprim) {
    std::vector<double> c(nprim);
    const double df = double_factorial(2 * L - 1);
    for (int i = 0; i < nprim; ++i) {
        const double num = std::pow(2.0, 2.0 * L + 1.5) * std::pow(exps[i], L + 1.5);
        const double den = std::pow(kPi, 1.5) * df;
        c[i] = coefs[i] * std::sqrt(num / den);
    }
    // same-centre self overlap of the component x^L: (pi/p)^1.5 (2L-1)!!/(2p)^L
    double norm2 = 0.0;
    for (int i = 0; i < nprim; ++i)
        for (int j = 0; j < nprim; ++j) {
            const double p = exps[i] + exps[j];
            norm2 += c[i] * c[j] * std::pow(kPi / p, 1.5) * df / std::pow(2.0 * p, L);
        }
    const double scale = 1.0 / std::sqrt(norm2);
    for (auto& v : c) v *= scale;
    return c;
}

// make_shell's per-component normalisation (shell_contract.cpp:9-39,
// shell_math.cpp:50-77): N(a, ang) = sqrt(2^(2L+1.5) a^(L+1.5) /
// (pi^1.5 prod(2l-1)!!)) and the same-centre metric from the 1-D shape
// table at PA = AB = 0.
double same_center_factor(int l, double p) {
    const int ltot = 2 * l, ncol = l + 1;
    std::vector<double> out(static_cast<std::size_t>(ltot + 1) * ncol, 0.0);
    out[0] = 1.0;
    if (ltot >= 1) out[ncol] = 0.0;
    for (int n = 1; n < ltot; ++n)
        out[(n + 1) * ncol] = 0.0 * out[n * ncol] + (static_cast<double>(n) / (2.0 * p)) * out[(n - 1) * ncol];
    for (int ib = 0; ib < l; ++ib)
        for (int ia = 0; ia <= ltot - ib - 1; ++ia)
            out[ia * ncol + ib + 1] = out[(ia + 1) * ncol + ib] + 0.0 * out[ia * ncol + ib];
    return out[l * (l + 1) + l];
}

std::vector<double> normalise_component(int lx, int ly, int lz, const double* exps, const double* coefs, int nprim) {
    const int L = lx + ly + lz;
    const double df = double_factorial(2 * lx - 1) * double_factorial(2 * ly - 1) * double_factorial(2 * lz - 1);
    std::vector<double> c(nprim);
    for (int i = 0; i < nprim; ++i) {
        const double num = std::pow(2.0, 2.0 * static_cast<double>(L) + 1.5) * std::pow(exps[i], static_cast<double>(L) + 1.5);
        const double den = std::pow(kPi, 1.5) * df;
        c[i] = coefs[i] * std::sqrt(num / den);
    }
    double norm2 = 0.0;
    for (int i = 0; i < nprim; ++i)
        for (int j = 0; j < nprim; ++j) {
            const double p = exps[i] + exps[j];
            const double metric = std::pow(kPi / p, 1.5) * same_center_factor(lx, p) * same_center_factor(ly, p) *
                                  same_center_factor(lz, p);
            norm2 += c[i] * c[j] * metric;
        }
    const double scale = 1.0 / std::sqrt(norm2);
    for (auto& v : c) v *= scale;
    return c;
}

void validate_shell(const double* center, int L, int nprim, const double* exps, const double* coefs) {
    for (int k = 0; k < 3; ++k)
        if (!finite_bits(center[k])) throw Error(-1, "eri_ao_tensor_hgp: shell centers must be finite.");
    if (L < 0) throw Error(-1, "eri_ao_tensor_hgp: Cartesian angular powers must be nonnegative.");
    if (L > kMaxL) throw Error(-1, "eri_ao_tensor_hgp: pure-spherical stream supports shell L=0..4.");
    if (nprim <= 0) throw Error(-1, "eri_ao_tensor_hgp: contracted shells need at least one primitive.");
    for (int i = 0; i < nprim; ++i)
        if (!finite_bits(exps[i]) || !(exps[i] > 0.0) || !finite_bits(coefs[i]))
            throw Error(-1,
                        "eri_ao_tensor_hgp: primitive exponents must be finite and positive and "
                        "coefficients must be finite.");
}

void finish_basis(Basis& b, int natom, const int* Z, const double* atom_xyz) {
    b.n_sph = 0;
    b.n_cart = 0;
    b.max_L = 0;
    b.max_nprim = 0;
    for (auto& s : b.shells) {
        s.sph_offset = b.n_sph;
        s.cart_offset = b.n_cart;
        b.n_sph += n_sph(s.L);
        b.n_cart += n_cart(s.L);
        b.max_L = std::max(b.max_L, s.L);
        b.max_nprim = std::max(b.max_nprim, s.nprim);
    }
    for (int a = 0; a < natom; ++a) {
        for (int k = 0; k < 3; ++k)
            if (!finite_bits(atom_xyz[3 * a + k])) throw Error(-1, "tlno_gpu: nuclear centres must be finite.");
        b.Z.push_back(Z[a]);
        b.atom_xyz.insert(b.atom_xyz.end(), atom_xyz + 3 * a, atom_xyz + 3 * a + 3);
    }
    // One-electron screening groups: equal L, centre and exponent list.
    b.onee_group.assign(b.shells.size(), -1);
    std::map<std::vector<double>, int> key_to_group;
    for (std::size_t i = 0; i < b.shells.size(); ++i) {
        const Shell& s = b.shells[i];
        std::vector<double> key = {double(s.L), s.center[0], s.center[1], s.center[2]};
        key.insert(key.end(), b.exps.begin() + s.prim_offset, b.exps.begin() + s.prim_offset + s.nprim);
        auto it = key_to_group.find(key);
        if (it == key_to_group.end()) {
            const int g = static_cast<int>(b.onee_group_rep.size());
            key_to_group.emplace(std::move(key), g);
            b.onee_group_rep.push_back(static_cast<int>(i));
            b.onee_group[i] = g;
        } else {
            b.onee_group[i] = it->second;
        }
    }
}

}  // namespace

Basis basis_from_raw(int n_shells, const double* centers, const int* L, const int* nprim,
                     const double* exps, const double* coefs, int natom, const int* Z,
                     const double* atom_xyz) {
    if (n_shells < 0 || natom < 0) throw Error(-1, "tlno_gpu: negative shell or atom count.");
    Basis b;
    std::size_t off = 0;
    for (int s = 0; s < n_shells; ++s) {
        validate_shell(centers + 3 * s, L[s], nprim[s], exps + off, coefs + off);
        Shell sh{};
        for (int k = 0; k < 3; ++k) sh.center[k] = centers[3 * s + k];
        sh.L = L[s];
        sh.nprim = nprim[s];
        sh.prim_offset = static_cast<int>(b.exps.size());
        sh.atom = -1;
        const std::vector<double> cxl = normalise_xl(L[s], exps + off, coefs + off, nprim[s]);
        const double inv_na = 1.0 / ang_norm(L[s], 0, 0);
        for (int i = 0; i < nprim[s]; ++i) {
            b.exps.push_back(exps[off + i]);
            b.c_radial.push_back(cxl[i] * inv_na);
        }
        b.comp_offset.push_back(static_cast<int>(b.comp_coef.size()));
        for (int x = L[s]; x >= 0; --x)
            for (int y = L[s] - x; y >= 0; --y) {
                const auto cc = normalise_component(x, y, L[s] - x - y, exps + off, coefs + off, nprim[s]);
                b.comp_coef.insert(b.comp_coef.end(), cc.begin(), cc.end());
            }
        b.shells.push_back(sh);
        off += static_cast<std::size_t>(nprim[s]);
    }
    finish_basis(b, natom, Z, atom_xyz);
    return b;
}

Basis basis_from_components(int n_comp, const double* centers, const int* ang, const int* nprim,
                            const double* exps, const double* coefs, int natom, const int* Z,
                            const double* atom_xyz) {
    if (n_comp < 0 || natom < 0) throw Error(-1, "tlno_gpu: negative component or atom count.");
    // Group components: same L and centre and the same radial contraction
    // (coefficient / N_ang equal to 32 ulp, exponents equal), first-appearance
    // order (rys_engine.ipp:1928-2035).
    struct Group {
        int L;
        double center[3];
        std::vector<double> e, crad;
        std::vector<int> seen;
        std::vector<std::vector<double>> comp;  // canonical component order
        int count = 0;
    };
    std::vector<Group> groups;
    std::size_t off = 0;
    for (int k = 0; k < n_comp; ++k) {
        const int lx = ang[3 * k], ly = ang[3 * k + 1], lz = ang[3 * k + 2];
        if (lx < 0 || ly < 0 || lz < 0)
            throw Error(-1, "eri_ao_tensor_hgp: Cartesian angular powers must be nonnegative.");
        const int Lk = lx + ly + lz;
        validate_shell(centers + 3 * k, Lk, nprim[k], exps + off, coefs + off);
        const double na = ang_norm(lx, ly, lz);
        std::vector<double> crad(nprim[k]);
        for (int i = 0; i < nprim[k]; ++i) crad[i] = coefs[off + i] / na;
        int gi = -1;
        for (std::size_t g = 0; g < groups.size(); ++g) {
            Group& G = groups[g];
            if (G.L != Lk || G.center[0] != centers[3 * k] || G.center[1] != centers[3 * k + 1] ||
                G.center[2] != centers[3 * k + 2] || static_cast<int>(G.e.size()) != nprim[k])
                continue;
            bool same = true;
            for (int i = 0; i < nprim[k] && same; ++i) {
                if (G.e[i] != exps[off + i]) same = false;
                const double l = G.crad[i], r = crad[i];
                const double sc = std::max(std::fabs(l), std::fabs(r));
                if (!(l == r || sc == 0.0 || std::fabs(l - r) <= 32.0 * 2.220446049250313e-16 * sc)) same = false;
            }
            if (same) { gi = static_cast<int>(g); break; }
        }
        if (gi < 0) {
            Group G;
            G.L = Lk;
            for (int c = 0; c < 3; ++c) G.center[c] = centers[3 * k + c];
            G.e.assign(exps + off, exps + off + nprim[k]);
            G.crad = crad;
            G.seen.assign(n_cart(Lk), 0);
            G.comp.assign(n_cart(Lk), {});
            groups.push_back(std::move(G));
            gi = static_cast<int>(groups.size()) - 1;
        }
        Group& G = groups[gi];
        const int dx = Lk - lx;
        const int local = dx * (dx + 1) / 2 + (dx - ly);
        if (G.seen[local])
            throw Error(-1, "eri_ao_tensor_hgp: duplicate or invalid Cartesian component inside a contracted shell.");
        G.seen[local] = 1;
        G.comp[local].assign(coefs + off, coefs + off + nprim[k]);
        ++G.count;
        off += static_cast<std::size_t>(nprim[k]);
    }
    Basis b;
    for (auto& G : groups) {
        if (G.count != n_cart(G.L))
            throw Error(-1, "eri_ao_tensor_hgp: each radial contraction must contain exactly one complete Cartesian shell.");
        Shell sh{};
        for (int c = 0; c < 3; ++c) sh.center[c] = G.center[c];
        sh.L = G.L;
        sh.nprim = static_cast<int>(G.e.size());
        sh.prim_offset = static_cast<int>(b.exps.size());
        sh.atom = -1;
        b.exps.insert(b.exps.end(), G.e.begin(), G.e.end());
        b.c_radial.insert(b.c_radial.end(), G.crad.begin(), G.crad.end());
        b.comp_offset.push_back(static_cast<int>(b.comp_coef.size()));
        for (const auto& cc : G.comp) b.comp_coef.insert(b.comp_coef.end(), cc.begin(), cc.end());
        b.shells.push_back(sh);
    }
    finish_basis(b, natom, Z, atom_xyz);
    return b;
}

}  // namespace tlno_gpu
