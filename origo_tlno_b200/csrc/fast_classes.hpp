// Classes with a compile-time ERI kernel (la >= lb, lc >= ld, bra class
// index >= ket class index): every class with shells up to d and the f
// classes with one f shell whose instantiation compiles in a few minutes
// (bra (fs), (fp) against kets up to (dp)/(fs), (fd) against (ss), (ps),
// (ds)).  The other f classes take the warp-per-quartet kernel.  Each class
// is compiled in its own translation unit (eri_fast_inst.cu with
// -DTLNO_FAST_ID=<index>).
#pragma once

#include <cuda_runtime.h>

#define TLNO_FAST_CLASSES(X) \
    X(0, 0, 0, 0, 0) \
    X(1, 1, 0, 0, 0) \
    X(2, 1, 0, 1, 0) \
    X(3, 1, 1, 0, 0) \
    X(4, 1, 1, 1, 0) \
    X(5, 1, 1, 1, 1) \
    X(6, 2, 0, 0, 0) \
    X(7, 2, 0, 1, 0) \
    X(8, 2, 0, 1, 1) \
    X(9, 2, 0, 2, 0) \
    X(10, 2, 1, 0, 0) \
    X(11, 2, 1, 1, 0) \
    X(12, 2, 1, 1, 1) \
    X(13, 2, 1, 2, 0) \
    X(14, 2, 1, 2, 1) \
    X(15, 2, 2, 0, 0) \
    X(16, 2, 2, 1, 0) \
    X(17, 2, 2, 1, 1) \
    X(18, 2, 2, 2, 0) \
    X(19, 2, 2, 2, 1) \
    X(20, 2, 2, 2, 2) \
    X(21, 3, 0, 0, 0) \
    X(22, 3, 0, 1, 0) \
    X(23, 3, 0, 1, 1) \
    X(24, 3, 0, 2, 0) \
    X(25, 3, 0, 2, 1) \
    X(26, 3, 0, 2, 2) \
    X(27, 3, 0, 3, 0) \
    X(28, 3, 1, 0, 0) \
    X(29, 3, 1, 1, 0) \
    X(30, 3, 1, 1, 1) \
    X(31, 3, 1, 2, 0) \
    X(32, 3, 1, 2, 1) \
    X(33, 3, 2, 0, 0) \
    X(34, 3, 2, 1, 0) \
    X(35, 3, 2, 2, 0)

#define TLNO_FAST_COUNT 36

namespace tlno_gpu {
namespace dev {
struct DevTables;
struct CartTable;
struct C2STable;
struct PlanView;
struct ClassLaunch;
}  // namespace dev

// Defined once per class by eri_fast_inst.cu.
#define TLNO_FAST_DECL(id, a, b, c, d)                                                          \
    void fast_upload_##id(const dev::DevTables&, const dev::CartTable&, const dev::C2STable&); \
    int fast_bras_##id();                                                                      \
    int fast_blocks_per_sm_##id(bool fp32);                                                    \
    void fast_launch_##id(bool fp32, const dev::PlanView&, const dev::ClassLaunch&, int grid, cudaStream_t s);
TLNO_FAST_CLASSES(TLNO_FAST_DECL)
#undef TLNO_FAST_DECL

inline int fast_class_index(int la, int lb, int lc, int ld) {
#define TLNO_FAST_MATCH(id, a, b, c, d) \
    if (la == a && lb == b && lc == c && ld == d) return id;
    TLNO_FAST_CLASSES(TLNO_FAST_MATCH)
#undef TLNO_FAST_MATCH
    return -1;
}

}  // namespace tlno_gpu
