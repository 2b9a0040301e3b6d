// TEST INFRASTRUCTURE ONLY -- never linked into the shipped library.
//
// C-ABI harness around the UNMODIFIED reference front end (the molecule
// reader benchmarks/common/molecule_io.cpp and the named-basis builder
// core/basis/basis_general.cpp with its get_*_params tables), compiled from
// the reference's own sources by oracle/build_ref.sh into
// oracle/_ref/libtlno_ref.so.  Only tests/ use it, as the checker of the
// engine's own front end (origo_tlno_b200/frontend.py).
#include <cstring>
#include <string>
#include <vector>

#include "benchmarks/common/molecule_io.hpp"
#include "core/basis/basis_general.hpp"
#include "core/basis/get_4_31g_params.hpp"
#include "core/basis/get_6_31g_d_params.hpp"
#include "core/basis/get_6_31g_dp_params.hpp"
#include "core/basis/get_6_31g_params.hpp"
#include "core/basis/get_def2_svp_params.hpp"
#include "core/basis/get_def2_tzvp_params.hpp"
#include "core/basis/get_sto3g_params.hpp"

namespace {
thread_local std::string g_err;

template <class F>
int guarded(F&& f) {
    try {
        f();
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
    } catch (...) {
        g_err = "unknown exception";
    }
    return -1;
}

}  // namespace

extern "C" {

const char* ref_frontend_last_error() { return g_err.c_str(); }

// read_inp_file (molecule_io.cpp:104-165): symbols as 8-byte NUL-padded
// records, coordinates in bohr.
int ref_read_inp(const char* path, int max_atoms, int* natom, char* symbols, double* coords, int* charge,
                 int* multiplicity) {
    return guarded([&] {
        const auto m = tlno::benchmarks::onee::read_inp_file(path);
        *natom = static_cast<int>(m.symbols.size());
        *charge = m.charge;
        *multiplicity = m.multiplicity;
        if (*natom > max_atoms) return;
        for (int a = 0; a < *natom; ++a) {
            std::memset(symbols + 8 * a, 0, 8);
            std::strncpy(symbols + 8 * a, m.symbols[a].c_str(), 7);
            for (int k = 0; k < 3; ++k) coords[3 * a + k] = m.coords_bohr[a][k];
        }
    });
}

// build_basis_general (basis_general.cpp:77-111) for a molecule given as
// symbols + bohr coordinates: the Cartesian component records
// (centre, angular triple, make_shell-normalised primitives), nuclear
// charges and the electron count.  Call with null arrays for the counts.
int ref_basis_general(int natom, const char* symbols, const double* coords, int charge, const char* basis,
                      int* n_components, int* n_prims, double* centers, int* ang, int* nprim, double* exps,
                      double* coefs, int* Z, int* electrons) {
    return guarded([&] {
        tlno::core::molecule::MoleculeSpec spec;
        spec.charge = charge;
        for (int a = 0; a < natom; ++a) {
            spec.symbols.emplace_back(symbols + 8 * a);
            spec.coords.push_back({coords[3 * a], coords[3 * a + 1], coords[3 * a + 2]});
        }
        const auto r = tlno::core::basis::build_basis_general(spec, tlno::core::basis::parse_basis_kind(basis));
        *n_components = static_cast<int>(r.basis.size());
        int np = 0;
        for (const auto& s : r.basis) np += static_cast<int>(s.primitives.size());
        *n_prims = np;
        if (electrons) *electrons = r.electron_count;
        if (!centers) return;
        int p = 0;
        for (std::size_t k = 0; k < r.basis.size(); ++k) {
            for (int a = 0; a < 3; ++a) {
                centers[3 * k + a] = r.basis[k].center[a];
                ang[3 * k + a] = r.basis[k].ang[a];
            }
            nprim[k] = static_cast<int>(r.basis[k].primitives.size());
            for (const auto& pr : r.basis[k].primitives) {
                exps[p] = pr.exponent;
                coefs[p] = pr.coefficient;
                ++p;
            }
        }
        for (int a = 0; a < natom; ++a) Z[a] = r.nuclear_charges[a];
    });
}

// The reference's raw per-element basis table (RawAtomBasis: one raw shell
// per Cartesian component, BSE coefficients before make_shell) of a basis
// kind name, for writing a basis file the engine's front end reads back.
// Call with null arrays for the counts.
int ref_raw_atom_basis(const char* symbol, const char* basis, int* charge, int* n_raw, int* n_prims, int* ang,
                       int* nprim, double* exps, double* coefs) {
    return guarded([&] {
        namespace b = tlno::core::basis;
        b::RawAtomBasis a;
        switch (b::parse_basis_kind(basis)) {
            case b::BasisKind::Sto3g: a = b::get_sto3g_params(symbol); break;
            case b::BasisKind::G431: a = b::get_4_31g_params(symbol); break;
            case b::BasisKind::G631: a = b::get_6_31g_params(symbol); break;
            case b::BasisKind::G631d: a = b::get_6_31g_d_params(symbol); break;
            case b::BasisKind::G631dp: a = b::get_6_31g_dp_params(symbol); break;
            case b::BasisKind::Def2SVP: a = b::get_def2_svp_params(symbol); break;
            case b::BasisKind::Def2TZVP: a = b::get_def2_tzvp_params(symbol); break;
        }
        *charge = a.charge;
        *n_raw = static_cast<int>(a.shells.size());
        int np = 0;
        for (const auto& s : a.shells) np += static_cast<int>(s.exponents.size());
        *n_prims = np;
        if (!ang) return;
        int p = 0;
        for (std::size_t k = 0; k < a.shells.size(); ++k) {
            for (int t = 0; t < 3; ++t) ang[3 * k + t] = a.shells[k].ang[t];
            nprim[k] = static_cast<int>(a.shells[k].exponents.size());
            for (std::size_t i = 0; i < a.shells[k].exponents.size(); ++i) {
                exps[p] = a.shells[k].exponents[i];
                coefs[p] = a.shells[k].coefficients[i];
                ++p;
            }
        }
    });
}

// parse_basis_kind (basis_general.cpp:48-75): 0 on a name it accepts.
int ref_parse_basis_kind(const char* name) {
    return guarded([&] { (void)tlno::core::basis::parse_basis_kind(name); });
}

}  // extern "C"
