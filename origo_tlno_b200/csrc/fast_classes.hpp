// Classes with a thread-per-quartet ERI kernel (la >= lb, lc >= ld, bra
// class index >= ket class index), chosen so that their contracted radial
// accumulators fit in registers.  Each class is compiled in its own
// translation unit (eri_fast_inst.cu with -DTLNO_FAST_ID=<index>).
#pragma once

#include <cuda_runtime.h>

#define TLNO_FAST_CLASSES(X) \
    X(0, 0, 0, 0, 0)         \
    X(1, 1, 0, 0, 0)         \
    X(2, 1, 0, 1, 0)         \
    X(3, 1, 1, 0, 0)         \
    X(4, 1, 1, 1, 0)         \
    X(5, 2, 0, 0, 0)         \
    X(6, 2, 0, 1, 0)         \
    X(7, 2, 0, 1, 1)         \
    X(8, 2, 0, 2, 0)         \
    X(9, 2, 1, 0, 0)         \
    X(10, 2, 2, 0, 0)

#define TLNO_FAST_COUNT 11

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
    void fast_launch_##id(bool fp32, const dev::PlanView&, const dev::ClassLaunch&, int grid,   \
                          int threads, cudaStream_t s);
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
