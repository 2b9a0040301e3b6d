// Host-side structures of the B200 integral engine: normalised shells, the
// shell-pair plan sorted into (La, Lb) classes by Schwarz bound, and the
// quartet-class schedule.  Device-resident mirrors live in DevicePlan.
#pragma once

#include <cstddef>
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include <cuda_runtime.h>

namespace tlno_gpu {

constexpr int kMaxL = 4;            // s..g per shell (reference: rys_engine.ipp:2374)
constexpr int kMaxPairClasses = 15; // (La >= Lb) for La, Lb <= 4
constexpr double kPi = 3.141592653589793238462643383279502884;

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

void cuda_check(cudaError_t e, const char* what);
#define TLNO_CUDA(call) ::tlno_gpu::cuda_check((call), #call)

inline int n_cart(int L) { return (L + 1) * (L + 2) / 2; }
inline int n_sph(int L) { return 2 * L + 1; }
inline int pair_class_of(int la, int lb) { return la * (la + 1) / 2 + lb; }  // la >= lb

// One contracted shell after normalisation.
struct Shell {
    double center[3];
    int L;
    int nprim;
    int prim_offset;            // into Basis::exps / c_radial
    int sph_offset;             // first spherical AO
    int cart_offset;            // first Cartesian AO
    int atom;                   // unused by the math, kept for diagnostics
};

struct Basis {
    std::vector<Shell> shells;
    std::vector<double> exps;
    // Radial contraction coefficient per primitive: the make_shell-normalised
    // coefficient of the (L,0,0) component divided by its angular factor
    // 1/sqrt((2L-1)!!); every Cartesian component c of the shell then has
    // coefficient c_radial * N_ang(c) (rys_engine.ipp:2044-2058).
    std::vector<double> c_radial;
    // Normalised coefficient of every Cartesian component (one-electron
    // path): comp_coef[comp_offset(shell) + c * nprim + p], computed with the
    // same operations as the reference's make_shell so one-electron
    // integrals agree to rounding.
    std::vector<double> comp_coef;
    std::vector<int> comp_offset;
    std::vector<int> Z;
    std::vector<double> atom_xyz;  // 3 per atom
    int n_sph = 0;
    int n_cart = 0;
    int max_L = 0;
    int max_nprim = 0;
    // One-electron screening groups (same L, centre and exponent list),
    // as the reference groups components (onee_matrices.cpp:47-94).
    std::vector<int> onee_group;           // per shell
    std::vector<int> onee_group_rep;       // representative shell per group
};

// Builds a basis from raw contracted shells (normalised like make_shell).
Basis basis_from_raw(int n_shells, const double* centers, const int* L,
                     const int* nprim, const double* exps, const double* coefs,
                     int natom, const int* Z, const double* atom_xyz);
// Builds a basis from per-Cartesian-component records that are already
// normalised (the reference's std::vector<Shell> layout).
Basis basis_from_components(int n_comp, const double* centers, const int* ang,
                            const int* nprim, const double* exps,
                            const double* coefs, int natom, const int* Z,
                            const double* atom_xyz);

// Primitive pair record used by the ERI kernels (48 bytes).
struct PrimPair {
    double p;      // alpha + beta
    double Px, Py, Pz;
    double w;      // exp(-alpha beta / p |AB|^2) c_a c_b / p (radial coefs)
    double invp;   // 1 / p
};

// Shell pair (oriented: L_A >= L_B) -- the reference's pair group
// (rys_engine.ipp:2449-2468).
struct ShellPair {
    int A, B;          // shell indices after orientation
    int prim_offset;   // into PrimPair list
    int nprim;
    int cls;           // pair class (La, Lb)
};

struct DeviceBuffer {
    void* ptr = nullptr;
    std::size_t bytes = 0;
    DeviceBuffer() = default;
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
    DeviceBuffer(DeviceBuffer&& o) noexcept : ptr(o.ptr), bytes(o.bytes) { o.ptr = nullptr; o.bytes = 0; }
    DeviceBuffer& operator=(DeviceBuffer&& o) noexcept {
        if (this != &o) { release(); ptr = o.ptr; bytes = o.bytes; o.ptr = nullptr; o.bytes = 0; }
        return *this;
    }
    ~DeviceBuffer() { release(); }
    void release();
    void alloc(std::size_t n);                 // no-op when already large enough
    template <class T> T* as() const { return static_cast<T*>(ptr); }
};

}  // namespace tlno_gpu
