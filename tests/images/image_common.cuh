// Shared by the test images: the launch convention of registered sm_100a images.
#pragma once
#include <stdint.h>

#include "parallax/kernel_abi.h"

// Device address of a stored host pointer into the arena (the reference's relocation,
// shaders/relocate.comp:14-28): dev_base + (p - host_base).
template <typename T>
__device__ __forceinline__ T* relocate(const parallax_launch_args& a, const T* host_p) {
    return reinterpret_cast<T*>(a.dev_base + (reinterpret_cast<uint64_t>(host_p) - a.host_base));
}

#define PARALLAX_FOR_EACH_INDEX(a, i)                                                    \
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < (a).count;    \
         i += (uint64_t)gridDim.x * blockDim.x)
