// Fused transform + reduce tile, linked at run time with a registered transform image.
//
// Reference: the transform_reduce and count_if funnels run two passes - a transform
// kernel writing f(x) for every element into a staging buffer, then a '+' reduce of that
// buffer (include/parallax/stdpar.hpp:245-293). Here the transform's per-element function
// (`parallax_elem`, exported by an image compiled as relocatable LTO-IR; see
// include/parallax/kernel_abi.h) is linked into this reduce tile by nvJitLink with
// link-time optimisation, so it is inlined and f(x) never leaves registers: one read of the
// input, no staging buffer written or read back.
//
// This file is not part of the runtime library's normal compile: the build turns it into
// an LTO-IR fatbin (sm_100a) that the library embeds, and it is linked only together with
// an image that defines parallax_elem.
//
// The sum is accumulated as the runtime's reduce accumulates it (fp32 in fp64, fp64 in
// fp64, integers in their unsigned type, wrapping): per-thread partial sums over a
// grid-stride walk, a warp-shuffle then shared-memory fold per block, per-block partials,
// and the last block to finish (atomic ticket) folds the partials in block order, so the
// result is the same for every run of a given count and grid.
#include <stdint.h>

extern "C" __device__ void parallax_elem(const void* in, void* out);

namespace {

constexpr int kBlock = 256;
constexpr int kUnroll = 8;  // independent element loads in flight per thread

template <typename A>
__device__ __forceinline__ A shfl_down(A v, int d) {
    return __shfl_down_sync(0xffffffffu, v, d);
}

template <typename A>
__device__ __forceinline__ A block_sum(A v) {
    __shared__ A s_warp[kBlock / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) v = v + shfl_down(v, d);
    if (lane == 0) s_warp[warp] = v;
    __syncthreads();
    A r = A(0);
    if (warp == 0) {
        r = lane < kBlock / 32 ? s_warp[lane] : A(0);
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) r = r + shfl_down(r, d);
    }
    __syncthreads();  // s_warp may be reused by the caller's next fold
    return r;  // valid in thread 0
}

// U: the transform's output type (the reduced type), A: its accumulator.
template <typename U, typename A>
__device__ __forceinline__ void xform_reduce(const unsigned char* __restrict__ in, uint64_t n,
                                             uint32_t in_size, A* __restrict__ partials,
                                             unsigned* __restrict__ ticket, U* __restrict__ out) {
    const uint64_t G = (uint64_t)gridDim.x * kBlock;
    uint64_t i = (uint64_t)blockIdx.x * kBlock + threadIdx.x;
    A acc = A(0);
    for (; i + (kUnroll - 1) * G < n; i += kUnroll * G) {
        U u[kUnroll];
#pragma unroll
        for (int k = 0; k < kUnroll; ++k) parallax_elem(in + (i + k * G) * in_size, &u[k]);
#pragma unroll
        for (int k = 0; k < kUnroll; ++k) acc = acc + (A)u[k];
    }
    for (; i < n; i += G) {
        U u;
        parallax_elem(in + i * in_size, &u);
        acc = acc + (A)u;
    }
    const A b = block_sum(acc);
    __shared__ bool s_last;
    if (threadIdx.x == 0) {
        partials[blockIdx.x] = b;
        __threadfence();
        s_last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    A f = A(0);
    for (unsigned j = threadIdx.x; j < gridDim.x; j += kBlock)
        f = f + *reinterpret_cast<volatile A*>(partials + j);
    f = block_sum(f);
    if (threadIdx.x == 0) {
        *out = (U)f;
        *ticket = 0;  // self-reset for the next launch on this workspace
    }
}

}  // namespace

#define PXB_XFORM_REDUCE(NAME, U, A)                                                        \
    extern "C" __global__ void __launch_bounds__(kBlock)                                    \
        NAME(const unsigned char* in, uint64_t n, uint32_t in_size, A* partials,            \
             unsigned* ticket, U* out) {                                                    \
        xform_reduce<U, A>(in, n, in_size, partials, ticket, out);                          \
    }

PXB_XFORM_REDUCE(pxb_xform_reduce_f32, float, double)
PXB_XFORM_REDUCE(pxb_xform_reduce_f64, double, double)
PXB_XFORM_REDUCE(pxb_xform_reduce_i32, int32_t, uint32_t)
PXB_XFORM_REDUCE(pxb_xform_reduce_i64, int64_t, uint64_t)
PXB_XFORM_REDUCE(pxb_xform_reduce_u32, uint32_t, uint32_t)
PXB_XFORM_REDUCE(pxb_xform_reduce_u64, uint64_t, uint64_t)
