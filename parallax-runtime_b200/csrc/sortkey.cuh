// Order-preserving key transforms shared by the merge sort (kernels/sort.cu) and the radix
// sort (kernels/radix.cu): keys are sorted as unsigned integers after to_key and restored
// with from_key. Signed integers flip the sign bit; IEEE floats flip all bits when negative
// and only the sign bit otherwise, which orders them by the IEEE total order (-0.0 before
// +0.0, NaNs by sign and payload at the ends).
#pragma once

#include <stdint.h>

namespace pxb {

// XF: 0 unsigned (identity), 1 signed integer, 2 IEEE float
template <typename K, int XF>
__device__ __forceinline__ K to_key(K b) {
    constexpr K sign = K(1) << (sizeof(K) * 8 - 1);
    if constexpr (XF == 1) return b ^ sign;
    if constexpr (XF == 2) return (b & sign) ? ~b : (b | sign);
    return b;
}
template <typename K, int XF>
__device__ __forceinline__ K from_key(K k) {
    constexpr K sign = K(1) << (sizeof(K) * 8 - 1);
    if constexpr (XF == 1) return k ^ sign;
    if constexpr (XF == 2) return (k & sign) ? (k ^ sign) : ~k;
    return k;
}

}  // namespace pxb
