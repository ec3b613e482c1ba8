// Built-in element-wise kernels with captures and in-kernel pointer relocation.
//
// Reference: compiler-emitted SPIR-V maps dispatched as ceil(n/256) groups with the
// closure bytes in a uniform buffer and the arena bases in the push block
// (src/kernel/kernel_launcher.cpp:450-817); stored host pointers are relocated with
// gpu = dev_base + (host - host_base) (shaders/relocate.comp:14-28).
//
// Here: grid-stride kernels sized to the SM count, closure bytes passed by value in the
// kernel's parameter bank, 16-byte record loads, and the same relocation formula.
//   saxpy_gather_f32  transform2 over 16-byte records {float x; uint32 pad; float* p}:
//                     y = a * x + *relocate(p), a = captures[0:4] as float. The multiply
//                     and add are separately rounded (no FMA contraction), so results are
//                     bit-identical to host float arithmetic a*x + *p.
//   affine_f32        x = a * x + b, captures {float a, float b}, in place or in -> out.
//   relocate_f32      v = v * 2 + 1 over the arena array whose HOST address is
//                     captures[0:8]: the pointer-relocation check of the reference test
//                     (tests/unit/test_physptr.cpp:95-122).
#include <stdint.h>
#include <string.h>

#include "../runtime.hpp"

namespace pxb {
namespace {

constexpr int kBlock = 256;

struct MapArgs {
    const void* in;
    void* out;
    uint64_t n;
    uint64_t host_base;
    uint64_t dev_base;
    uint64_t host_end;          // end of the mapped arena range (host addresses)
    float a, b;
    uint64_t ptr;
    volatile int32_t* err;
};

// A stored pointer must point into the mapped arena (and be 4-byte aligned) before it is
// relocated; anything else is recorded as an error and skipped, never dereferenced.
__device__ __forceinline__ bool in_arena(const MapArgs& a, uint64_t p, uint64_t bytes) {
    return p >= a.host_base && p + bytes <= a.host_end && (p & 3u) == 0;
}

__device__ __forceinline__ const float* relocate(uint64_t host_ptr, uint64_t host_base,
                                                 uint64_t dev_base) {
    return reinterpret_cast<const float*>(dev_base + (host_ptr - host_base));
}

__global__ void __launch_bounds__(kBlock) k_saxpy_gather(MapArgs a) {
    const uint64_t G = (uint64_t)gridDim.x * kBlock;
    const uint4* rec = static_cast<const uint4*>(a.in);
    float* y = static_cast<float*>(a.out);
    for (uint64_t i = (uint64_t)blockIdx.x * kBlock + threadIdx.x; i < a.n; i += G) {
        const uint4 r = ldg_stream16(rec + i);
        const float x = __uint_as_float(r.x);
        const uint64_t p = (uint64_t)r.z | ((uint64_t)r.w << 32);
        if (!in_arena(a, p, 4)) {
            *a.err = 4;
            y[i] = __int_as_float(0x7fc00000);
            continue;
        }
        const float g = __ldg(relocate(p, a.host_base, a.dev_base));
        y[i] = __fadd_rn(__fmul_rn(a.a, x), g);
    }
}

__global__ void __launch_bounds__(kBlock) k_affine(MapArgs a) {
    const uint64_t G = (uint64_t)gridDim.x * kBlock;
    const float* x = static_cast<const float*>(a.in);
    float* y = static_cast<float*>(a.out);
    for (uint64_t i = (uint64_t)blockIdx.x * kBlock + threadIdx.x; i < a.n; i += G)
        y[i] = __fadd_rn(__fmul_rn(a.a, x[i]), a.b);
}

__global__ void __launch_bounds__(kBlock) k_relocate(MapArgs a) {
    const uint64_t G = (uint64_t)gridDim.x * kBlock;
    float* v = const_cast<float*>(relocate(a.ptr, a.host_base, a.dev_base));
    for (uint64_t i = (uint64_t)blockIdx.x * kBlock + threadIdx.x; i < a.n; i += G)
        v[i] = __fadd_rn(__fmul_rn(v[i], 2.0f), 1.0f);
}

unsigned grid_for(uint64_t n) {
    uint64_t blocks = (n + kBlock - 1) / kBlock;
    const uint64_t cap = (uint64_t)device_info().sm_count * 8;
    if (blocks > cap) blocks = cap;
    return blocks ? (unsigned)blocks : 1u;
}

}  // namespace

bool launch_map(Workspace& ws, MapOp op, const void* d_in, void* d_out, size_t n,
                const void* captures, size_t capture_size) {
    MapArgs a;
    memset(&a, 0, sizeof a);
    a.in = d_in;
    a.out = d_out;
    a.n = n;
    a.host_base = arena_host_base();
    a.dev_base = arena_dev_base();
    a.host_end = a.host_base + arena_mapped_bytes();
    a.err = &ws.d_slot->spin_error;
    const unsigned char* c = static_cast<const unsigned char*>(captures);
    cudaStream_t s = ws.stream();
    switch (op) {
        case MapOp::SAXPY_GATHER_F32:
            if (capture_size < 4 || !c) break;
            memcpy(&a.a, c, 4);
            {
                ProfScope prof(ws, "k_saxpy_gather", 24 * (uint64_t)n);
                k_saxpy_gather<<<grid_for(n), kBlock, 0, s>>>(a);
            }
            count_launch();
            return cuda_ok(cudaGetLastError(), "k_saxpy_gather launch");
        case MapOp::AFFINE_F32:
            if (capture_size < 8 || !c) break;
            memcpy(&a.a, c, 4);
            memcpy(&a.b, c + 4, 4);
            k_affine<<<grid_for(n), kBlock, 0, s>>>(a);
            count_launch();
            return cuda_ok(cudaGetLastError(), "k_affine launch");
        case MapOp::DOUBLE_PLUS_ONE_F32:
            if (capture_size < 8 || !c) break;
            memcpy(&a.ptr, c, 8);
            {
                ArenaBlock blk;
                const void* hp = reinterpret_cast<const void*>(a.ptr);
                const uint64_t off = a.ptr - a.host_base;
                if (!arena_find(hp, &blk) || off + 4 * (uint64_t)n > blk.offset + blk.size ||
                    (a.ptr & 3u)) {
                    set_error(PARALLAX_ERR_INVALID_ARGUMENT,
                              "relocate_f32: captured range is not inside one arena block");
                    return false;
                }
            }
            k_relocate<<<grid_for(n), kBlock, 0, s>>>(a);
            count_launch();
            return cuda_ok(cudaGetLastError(), "k_relocate launch");
        default:
            set_error(PARALLAX_ERR_INVALID_HANDLE, "map: not a built-in map kernel");
            return false;
    }
    set_error(PARALLAX_ERR_INVALID_ARGUMENT, "map: captures too small for this kernel");
    return false;
}

}  // namespace pxb
