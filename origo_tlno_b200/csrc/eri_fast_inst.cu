// One thread-per-quartet ERI class, selected at compile time by
// -DTLNO_FAST_ID=<index into TLNO_FAST_CLASSES> (see fast_classes.hpp); the
// build compiles this file once per class so the instantiations build in
// parallel.
#include <cuda_runtime.h>

#include "fast_classes.hpp"
#include "device_common.cuh"
#include "eri_fast.cuh"
#include "tables.hpp"

#ifndef TLNO_FAST_ID
#error "TLNO_FAST_ID must be defined"
#endif

namespace tlno_gpu {

// Dynamic shared memory: the row-exchange buffer of a sliced class, the FP32
// Rys interval polynomials in the FP32 kernels with N <= 3, and the per-tile
// density slots of the bra-group classes.
#define TLNO_FAST_IMPL(id, a, b, c, d)                                                                  \
    static int fast_smem_##id(bool fp32) {                                                              \
        constexpr int n = dev::fast_roots<a, b, c, d>();                                                \
        int bytes = dev::fast_smem_bytes<a, b, c, d>();                                                 \
        if (fp32 && n <= kRys32MaxN) bytes += rys32_intervals(n) * (kRys32Deg + 1) * 2 * n * 4;         \
        bytes += dev::fast_pre_bytes<a, b, c, d>(fp32);                                                 \
        return bytes;                                                                                   \
    }                                                                                                   \
    void fast_upload_##id(const dev::DevTables& t, const dev::CartTable& ct, const dev::C2STable& cs) {  \
        dev::upload_constant_tables(t, ct, cs);                                                         \
        cudaFuncSetAttribute(dev::eri_fast_jk_kernel<double, a, b, c, d>,                               \
                             cudaFuncAttributeMaxDynamicSharedMemorySize, fast_smem_##id(false));       \
        cudaFuncSetAttribute(dev::eri_fast_jk_kernel<float, a, b, c, d>,                                \
                             cudaFuncAttributeMaxDynamicSharedMemorySize, fast_smem_##id(true));        \
    }                                                                                                   \
    int fast_bras_##id() { return dev::fast_bras<a, b, c, d>(); }                                       \
    int fast_blocks_per_sm_##id(bool fp32) {                                                            \
        constexpr int threads = 32 * dev::fast_warps<a, b, c, d>();                                     \
        int n = 0;                                                                                      \
        if (fp32)                                                                                       \
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, dev::eri_fast_jk_kernel<float, a, b, c, d>, \
                                                          threads, fast_smem_##id(true));               \
        else                                                                                            \
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, dev::eri_fast_jk_kernel<double, a, b, c, d>, \
                                                          threads, fast_smem_##id(false));              \
        return n > 0 ? n : 1;                                                                           \
    }                                                                                                   \
    void fast_launch_##id(bool fp32, const dev::PlanView& pv, const dev::ClassLaunch& cl, int grid,     \
                          cudaStream_t s) {                                                             \
        constexpr int threads = 32 * dev::fast_warps<a, b, c, d>();                                     \
        if (fp32)                                                                                       \
            dev::eri_fast_jk_kernel<float, a, b, c, d><<<grid, threads, fast_smem_##id(true), s>>>(pv, cl); \
        else                                                                                            \
            dev::eri_fast_jk_kernel<double, a, b, c, d><<<grid, threads, fast_smem_##id(false), s>>>(pv, cl); \
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
#if TLNO_FAST_ID == 11
#define TLNO_FAST_IF_11(x) x
#else
#define TLNO_FAST_IF_11(x)
#endif
#if TLNO_FAST_ID == 12
#define TLNO_FAST_IF_12(x) x
#else
#define TLNO_FAST_IF_12(x)
#endif
#if TLNO_FAST_ID == 13
#define TLNO_FAST_IF_13(x) x
#else
#define TLNO_FAST_IF_13(x)
#endif
#if TLNO_FAST_ID == 14
#define TLNO_FAST_IF_14(x) x
#else
#define TLNO_FAST_IF_14(x)
#endif
#if TLNO_FAST_ID == 15
#define TLNO_FAST_IF_15(x) x
#else
#define TLNO_FAST_IF_15(x)
#endif
#if TLNO_FAST_ID == 16
#define TLNO_FAST_IF_16(x) x
#else
#define TLNO_FAST_IF_16(x)
#endif
#if TLNO_FAST_ID == 17
#define TLNO_FAST_IF_17(x) x
#else
#define TLNO_FAST_IF_17(x)
#endif
#if TLNO_FAST_ID == 18
#define TLNO_FAST_IF_18(x) x
#else
#define TLNO_FAST_IF_18(x)
#endif

#if TLNO_FAST_ID == 19
#define TLNO_FAST_IF_19(x) x
#else
#define TLNO_FAST_IF_19(x)
#endif
#if TLNO_FAST_ID == 20
#define TLNO_FAST_IF_20(x) x
#else
#define TLNO_FAST_IF_20(x)
#endif

#if TLNO_FAST_ID == 21
#define TLNO_FAST_IF_21(x) x
#else
#define TLNO_FAST_IF_21(x)
#endif
#if TLNO_FAST_ID == 22
#define TLNO_FAST_IF_22(x) x
#else
#define TLNO_FAST_IF_22(x)
#endif
#if TLNO_FAST_ID == 23
#define TLNO_FAST_IF_23(x) x
#else
#define TLNO_FAST_IF_23(x)
#endif
#if TLNO_FAST_ID == 24
#define TLNO_FAST_IF_24(x) x
#else
#define TLNO_FAST_IF_24(x)
#endif
#if TLNO_FAST_ID == 25
#define TLNO_FAST_IF_25(x) x
#else
#define TLNO_FAST_IF_25(x)
#endif
#if TLNO_FAST_ID == 26
#define TLNO_FAST_IF_26(x) x
#else
#define TLNO_FAST_IF_26(x)
#endif
#if TLNO_FAST_ID == 27
#define TLNO_FAST_IF_27(x) x
#else
#define TLNO_FAST_IF_27(x)
#endif
#if TLNO_FAST_ID == 28
#define TLNO_FAST_IF_28(x) x
#else
#define TLNO_FAST_IF_28(x)
#endif
#if TLNO_FAST_ID == 29
#define TLNO_FAST_IF_29(x) x
#else
#define TLNO_FAST_IF_29(x)
#endif
#if TLNO_FAST_ID == 30
#define TLNO_FAST_IF_30(x) x
#else
#define TLNO_FAST_IF_30(x)
#endif
#if TLNO_FAST_ID == 31
#define TLNO_FAST_IF_31(x) x
#else
#define TLNO_FAST_IF_31(x)
#endif
#if TLNO_FAST_ID == 32
#define TLNO_FAST_IF_32(x) x
#else
#define TLNO_FAST_IF_32(x)
#endif
#if TLNO_FAST_ID == 33
#define TLNO_FAST_IF_33(x) x
#else
#define TLNO_FAST_IF_33(x)
#endif
#if TLNO_FAST_ID == 34
#define TLNO_FAST_IF_34(x) x
#else
#define TLNO_FAST_IF_34(x)
#endif
#if TLNO_FAST_ID == 35
#define TLNO_FAST_IF_35(x) x
#else
#define TLNO_FAST_IF_35(x)
#endif

TLNO_FAST_CLASSES(TLNO_FAST_SELECT)

}  // namespace tlno_gpu
