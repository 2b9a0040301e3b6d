// Host-visible launch wrappers of the device code in kernels.cu.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace tlno_gpu {
namespace dev {
struct PlanView;
struct ClassLaunch;
struct OneeLaunch;
}  // namespace dev

// Uploads the constant tables (Boys, Rys, Cartesian, cart->sph) for the
// current device; idempotent per device.
void ensure_device_tables();

// Shared-memory bytes per warp of the generic kernel for a class.
int generic_warp_bytes(int la, int lb, int lc, int ld);
// Builds the pair projectors of every pair with an offset >= 0.
void launch_pair_projectors(const int* pair_A, const int* pair_B, const double* shell_xyz, const int* shell_L,
                            const long long* off, int n_pairs, double* out, cudaStream_t s);

void launch_eri_store(const dev::PlanView& pv, const dev::ClassLaunch& cl, cudaStream_t s);
void launch_eri_schwarz(const dev::PlanView& pv, const dev::ClassLaunch& cl, cudaStream_t s);
void launch_eri_jk_generic(const dev::PlanView& pv, const dev::ClassLaunch& cl, bool fp32,
                           int warps, int grid, cudaStream_t s);
// Thread-per-quartet kernels for the classes that have one; returns false
// when the class has no specialised kernel.
bool launch_eri_jk_fast(const dev::PlanView& pv, const dev::ClassLaunch& cl, bool fp32,
                        int grid, cudaStream_t s);
bool has_fast_kernel(int la, int lb, int lc, int ld);
// Bra pairs per CTA of the compile-time kernel of a class (its schedule's
// block height).
int fast_kernel_bras(int la, int lb, int lc, int ld);

void launch_onee(const dev::OneeLaunch& L, cudaStream_t s);
// out = (X + X^T) / 2 for `count` stacked M x M blocks (offsets per block).
void launch_symmetrize(double* X, const long long* offsets, const int* dims, int count, int max_m,
                       cudaStream_t s);
void launch_symmetrize_single(double* X, int M, cudaStream_t s);
// *out = max |x_i| over n elements.
void launch_absmax(const double* x, long long n, double* out, cudaStream_t s);
// max|x| into *out and the FP32 copy x32 of x, one pass.
void launch_absmax_f32(const double* x, long long n, double* out, float* x32, cudaStream_t s);
// Density contract check: bit 1 = non-finite entry, bit 2 = asymmetric
// beyond 128 eps * max(1, |Dij|, |Dji|) (direct_build.ipp:25-96).
void launch_validate_density(const double* D, int M, unsigned int* status, cudaStream_t s);
// CVHF density tables per molecule: blk[off[mol] + i * ns + j] = max |D| over
// shell block (i, j) and its transpose, rho_max[mol] = max |D| (zeroed here).
// Single molecule: null per-molecule arrays, M1 / ns1 give the sizes.
void launch_density_blocks(const double* D, const long long* mat_off, const int* mol_M, int M1, const int* shell_sph,
                           const int* shell_L, const int* mol_shell_off, const int* mol_ns, int ns1, int n_mol,
                           long long max_entries, const long long* blk_off, double* blk, double* rho_max,
                           cudaStream_t s);
// delta = Dn - Dp with the incremental state's checks: status bit 1 = Dn
// non-finite, 2 = delta non-finite, 4 = delta nonzero somewhere; *dmax =
// max |delta| (max |Dn| when Dp is null; delta then untouched).
void launch_density_delta(const double* Dn, const double* Dp, double* delta, long long n, unsigned int* status,
                          double* dmax, cudaStream_t s);
// out = Gp + dG (or dG when Gp is null); status bit 1 = dG non-finite,
// 2 = out non-finite.
void launch_g_accumulate(const double* Gp, const double* dG, double* out, long long n, unsigned int* status,
                         cudaStream_t s);
// G = J - K / 2 over n elements.
void launch_combine_g(const double* J, const double* K, double* G, long long n, cudaStream_t s);
// Dependent-chain FMA throughput probe: returns TFLOP/s.
double measure_fma_peak(bool fp32);
void launch_boys_test(const double* x, int n, int maxn, double* out, cudaStream_t s);
void launch_rys_test(const double* t, int n, int nroots, int fp32, double* roots, double* weights,
                     cudaStream_t s);

}  // namespace tlno_gpu
