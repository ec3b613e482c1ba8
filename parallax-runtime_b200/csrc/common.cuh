// Shared device-side building blocks for the sm_100a primitive kernels: element types,
// 16-byte streaming loads, warp/block reductions, and acquire/release flag access used
// by the single-pass (decoupled look-back) kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>

namespace pxb {

// Mapped error-word code of the segment planner: offsets not non-decreasing within
// [0, count] (in-kernel wait timeouts use small positive codes).
constexpr int32_t kErrSegmentOffsets = 0x5e90;
// Mapped error-word code of the merge passes: a tile's two input spans on the merge path
// were inconsistent (only possible if a run was not sorted); the tile is skipped instead of
// staging outside its shared-memory buffer.
constexpr int32_t kErrMergeSpan = 0x5e91;
// Mapped error-word code of the radix passes: a CTA claimed a tile beyond the array or
// computed an output position outside it (only possible if a look-back word was corrupt);
// the access is skipped.
constexpr int32_t kErrRadixRange = 0x5e92;

// x % m == r for 32-bit integers with C semantics (the remainder takes the sign of x),
// dividing |x| by |m| as an invariant divisor: one multiply-high and two shifts
// (Granlund & Montgomery 1994, "Division by invariant integers using multiplication",
// Fig. 4.1: q = (t + ((n - t) >> sh1)) >> sh2, t = mulhi(magic, n)). am == 0 stands for a
// modulus that is zero in the element type; nothing matches it.
struct FastMod32 {
    uint32_t am = 0, magic = 0, sh1 = 0, sh2 = 0;
    // zero-remainder test (Granlund and Montgomery 1994, section 9): d = odd * 2^tz divides n
    // iff rotr(n * odd^-1 mod 2^32, tz) <= floor((2^32 - 1) / d)
    uint32_t inv = 0, tz = 0, lim = 0;
    static FastMod32 make(int64_t m) {  // m already converted to the element type
        FastMod32 f;
        const uint64_t d = (uint64_t)(m < 0 ? -m : m);
        if (d == 0 || d > 0xffffffffull) return f;
        uint32_t l = 0;
        while (l < 32 && (1ull << l) < d) ++l;  // l = ceil(log2 d)
        const unsigned __int128 num =
            ((unsigned __int128)1 << 32) * (((unsigned __int128)1 << l) - d);
        f.am = (uint32_t)d;
        f.magic = (uint32_t)(num / d + 1);
        f.sh1 = l < 1 ? l : 1;
        f.sh2 = l > 1 ? l - 1 : 0;
        uint32_t odd = (uint32_t)d;
        while (!(odd & 1u)) {
            odd >>= 1;
            ++f.tz;
        }
        uint32_t inv = odd;  // Newton iteration doubles the correct low bits: 3 -> 48
        for (int i = 0; i < 4; ++i) inv *= 2u - odd * inv;
        f.inv = inv;
        f.lim = 0xffffffffu / (uint32_t)d;
        return f;
    }
    // d divides n (am != 0)
    __device__ __forceinline__ bool divides(uint32_t n) const {
        const uint32_t q = n * inv;
        return __funnelshift_r(q, q, tz) <= lim;
    }
    __device__ __forceinline__ uint32_t rem(uint32_t n) const {
        const uint32_t t = __umulhi(magic, n);
        const uint32_t q = (t + ((n - t) >> sh1)) >> sh2;
        return n - q * am;
    }
    // x % m == 0 (C semantics: the sign of x does not matter)
    template <typename T>
    __device__ __forceinline__ bool eq0(T x) const {
        static_assert(sizeof(T) == 4, "32-bit integers");
        if constexpr (T(-1) < T(0)) {  // |INT_MIN| = 2^31 as unsigned
            return am != 0 && divides(x < T(0) ? 0u - (uint32_t)x : (uint32_t)x);
        } else {
            return am != 0 && divides((uint32_t)x);
        }
    }
    template <typename T>
    __device__ __forceinline__ bool eq(T x, T r) const {
        static_assert(sizeof(T) == 4, "32-bit integers");
        if (am == 0) return false;
        if constexpr (T(-1) < T(0)) {  // signed
            const bool neg = x < T(0);
            const uint32_t ra = rem(neg ? 0u - (uint32_t)x : (uint32_t)x);
            return (neg ? -(int64_t)ra : (int64_t)ra) == (int64_t)r;
        } else {
            return rem((uint32_t)x) == (uint32_t)r;
        }
    }
};

enum class DType : int { F32 = 0, F64 = 1, I32 = 2, I64 = 3, U32 = 4, U64 = 5, INVALID = -1 };

inline __host__ __device__ size_t dtype_size(DType t) {
    return (t == DType::F64 || t == DType::I64 || t == DType::U64) ? 8 : 4;
}
inline __host__ __device__ bool dtype_is_float(DType t) {
    return t == DType::F32 || t == DType::F64;
}

template <typename T> constexpr DType dtype_of();
template <> constexpr DType dtype_of<float>() { return DType::F32; }
template <> constexpr DType dtype_of<double>() { return DType::F64; }
template <> constexpr DType dtype_of<int32_t>() { return DType::I32; }
template <> constexpr DType dtype_of<int64_t>() { return DType::I64; }
template <> constexpr DType dtype_of<uint32_t>() { return DType::U32; }
template <> constexpr DType dtype_of<uint64_t>() { return DType::U64; }

// Accumulator used by '+' reductions and scans: fp32 data accumulates in fp64 (so a
// 2^28-element sum or prefix stays within 1e-5 of an fp64 oracle); integers accumulate
// in the unsigned type of the same width, i.e. two's-complement wrap-around, which is
// exact in any association order.
template <typename T> struct SumAcc;
template <> struct SumAcc<float> { using type = double; };
template <> struct SumAcc<double> { using type = double; };
template <> struct SumAcc<int32_t> { using type = uint32_t; };
template <> struct SumAcc<uint32_t> { using type = uint32_t; };
template <> struct SumAcc<int64_t> { using type = uint64_t; };
template <> struct SumAcc<uint64_t> { using type = uint64_t; };

// ---- 16-byte streaming global loads ---------------------------------------------------
// Read-only, no L1 allocation: every input byte of these kernels is touched once.
__device__ __forceinline__ uint4 ldg_stream16(const void* p) {
    uint4 r;
    asm volatile("ld.global.nc.L1::no_allocate.L2::256B.v4.u32 {%0,%1,%2,%3}, [%4];"
                 : "=r"(r.x), "=r"(r.y), "=r"(r.z), "=r"(r.w)
                 : "l"(p));
    return r;
}
// Streaming store: evict-first, the output is not re-read by this kernel.
__device__ __forceinline__ void stg_stream16(void* p, uint4 v) {
    asm volatile("st.global.cs.v4.u32 [%0], {%1,%2,%3,%4};" ::"l"(p), "r"(v.x), "r"(v.y),
                 "r"(v.z), "r"(v.w)
                 : "memory");
}

// ---- gpu-scope acquire/release on status words ----------------------------------------
__device__ __forceinline__ uint32_t ld_acquire_u32(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_u32(uint32_t* p, uint32_t v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void nanosleep_ns(unsigned ns) {
    asm volatile("nanosleep.u32 %0;" ::"r"(ns));
}

// ---- warp primitives -----------------------------------------------------------------
template <typename T>
__device__ __forceinline__ T shfl_up(T v, int d) {
    return __shfl_up_sync(0xffffffffu, v, d);
}
template <typename T>
__device__ __forceinline__ T shfl_xor(T v, int d) {
    return __shfl_xor_sync(0xffffffffu, v, d);
}
template <typename T>
__device__ __forceinline__ T shfl_idx(T v, int src) {
    return __shfl_sync(0xffffffffu, v, src);
}

struct OpSum {
    template <typename A> __device__ __forceinline__ A operator()(A a, A b) const { return a + b; }
};
struct OpMax {
    template <typename A> __device__ __forceinline__ A operator()(A a, A b) const {
        return b > a ? b : a;
    }
    __device__ __forceinline__ float operator()(float a, float b) const { return fmaxf(a, b); }
    __device__ __forceinline__ double operator()(double a, double b) const { return fmax(a, b); }
};
struct OpMin {
    template <typename A> __device__ __forceinline__ A operator()(A a, A b) const {
        return b < a ? b : a;
    }
    __device__ __forceinline__ float operator()(float a, float b) const { return fminf(a, b); }
    __device__ __forceinline__ double operator()(double a, double b) const { return fmin(a, b); }
};

template <typename A, typename Op>
__device__ __forceinline__ A warp_reduce(A v, Op op) {
#pragma unroll
    for (int d = 16; d >= 1; d >>= 1) v = op(v, shfl_xor(v, d));
    return v;
}

// Inclusive warp scan (Kogge-Stone over 32 lanes).
template <typename A, typename Op>
__device__ __forceinline__ A warp_inclusive_scan(A v, Op op) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        A u = shfl_up(v, d);
        if (lane >= d) v = op(u, v);
    }
    return v;
}

}  // namespace pxb
