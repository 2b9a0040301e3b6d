// Launch descriptors and J/K digestion shared by the ERI kernels.
#pragma once

#include "device_common.cuh"
#include "launch_types.hpp"

namespace tlno_gpu {
namespace dev {

enum Mode { kStore = 0, kSchwarz = 1, kJK = 2 };

// Bra-block index of a linear tile via binary search in the prefix array.
__device__ __forceinline__ int find_block(const int* prefix, int n_blocks, int tile) {
    int lo = 0, hi = n_blocks - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(prefix + mid) <= tile) lo = mid; else hi = mid - 1;
    }
    return lo;
}

}  // namespace dev
}  // namespace tlno_gpu
