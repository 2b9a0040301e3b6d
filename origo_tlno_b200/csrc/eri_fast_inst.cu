// One thread-per-quartet ERI class, selected at compile time by
// -DTLNO_FAST_ID=<index into TLNO_FAST_CLASSES> (see fast_classes.hpp); the
// build compiles this file once per class so the instantiations build in
// parallel.
#include <cuda_runtime.h>

#include "fast_classes.hpp"
#include "device_common.cuh"
#include "eri_fast.cuh"

#ifndef TLNO_FAST_ID
#error "TLNO_FAST_ID must be defined"
#endif

namespace tlno_gpu {

#define TLNO_FAST_IMPL(id, a, b, c, d)                                                                 \
    void fast_upload_##id(const dev::DevTables& t, const dev::CartTable& ct, const dev::C2STable& cs) { \
        dev::upload_constant_tables(t, ct, cs);                                                        \
    }                                                                                                  \
    void fast_launch_##id(bool fp32, const dev::PlanView& pv, const dev::ClassLaunch& cl, int grid,    \
                          int threads, cudaStream_t s) {                                               \
        if (fp32)                                                                                      \
            dev::eri_fast_jk_kernel<float, a, b, c, d><<<grid, threads, 0, s>>>(pv, cl);               \
        else                                                                                           \
            dev::eri_fast_jk_kernel<double, a, b, c, d><<<grid, threads, 0, s>>>(pv, cl);              \
    }

#define TLNO_FAST_SELECT(id, a, b, c, d) \
    TLNO_FAST_IF_##id(TLNO_FAST_IMPL(id, a, b, c, d))

#if TLNO_FAST_ID == 0
#define TLNO_FAST_IF_0(x) x
#else
#define TLNO_FAST_IF_0(x)
#endif
#if TLNO_FAST_ID == 1
#define TLNO_FAST_IF_1(x) x
#else
#define TLNO_FAST_IF_1(x)
#endif
#if TLNO_FAST_ID == 2
#define TLNO_FAST_IF_2(x) x
#else
#define TLNO_FAST_IF_2(x)
#endif
#if TLNO_FAST_ID == 3
#define TLNO_FAST_IF_3(x) x
#else
#define TLNO_FAST_IF_3(x)
#endif
#if TLNO_FAST_ID == 4
#define TLNO_FAST_IF_4(x) x
#else
#define TLNO_FAST_IF_4(x)
#endif
#if TLNO_FAST_ID == 5
#define TLNO_FAST_IF_5(x) x
#else
#define TLNO_FAST_IF_5(x)
#endif
#if TLNO_FAST_ID == 6
#define TLNO_FAST_IF_6(x) x
#else
#define TLNO_FAST_IF_6(x)
#endif
#if TLNO_FAST_ID == 7
#define TLNO_FAST_IF_7(x) x
#else
#define TLNO_FAST_IF_7(x)
#endif
#if TLNO_FAST_ID == 8
#define TLNO_FAST_IF_8(x) x
#else
#define TLNO_FAST_IF_8(x)
#endif
#if TLNO_FAST_ID == 9
#define TLNO_FAST_IF_9(x) x
#else
#define TLNO_FAST_IF_9(x)
#endif
#if TLNO_FAST_ID == 10
#define TLNO_FAST_IF_10(x) x
#else
#define TLNO_FAST_IF_10(x)
#endif

TLNO_FAST_CLASSES(TLNO_FAST_SELECT)

}  // namespace tlno_gpu
