// Tile staging shared by the single-pass scan and compaction kernels.
//
// A tile is NSUB sub-tiles of kBlock x ITEMS elements. One thread issues one 1-D bulk copy
// (cp.async.bulk into the CTA's own shared memory) per sub-tile, each completing on its own
// mbarrier, so work starts when the first sub-tile lands and the whole tile's bytes are in
// flight at once. The bulk-copied part of a tile is its 16-byte-aligned prefix; the ragged
// end of the last tile and the padding up to the tile size are filled with plain loads
// (padding = T(0)) by the whole CTA.
//
// The persistent kernels keep two tile buffers per CTA: while tile i is processed out of
// one buffer, the bulk copies of the CTA's next tile are already filling the other.
// Tiles are claimed from an atomic counter right before their copies are issued, and a
// CTA processes its claims in order; the lowest unfinished tile is therefore always the
// one its owner is processing, and it only waits on lower, finished tiles, so look-back
// waits end whatever CTAs happen to be resident.
#pragma once

#include <mutex>

#include "common.cuh"
#include "lookback.cuh"
#include "tma.cuh"

namespace pxb {

// Elements of a tile covered by bulk copies: its 16-byte-aligned prefix.
template <typename T>
__device__ __forceinline__ uint32_t bulk_elems(uint32_t cnt) {
    return (uint32_t)((cnt * sizeof(T)) / 16 * 16 / sizeof(T));
}

// Issued by ONE thread: the bulk copies of one tile, one per sub-tile, each arriving on
// bars[s]. Sub-tiles with nothing to copy complete immediately.
template <typename T, int SUB, int NSUB>
__device__ __forceinline__ void issue_tile(T* buf, uint64_t* bars, const T* in, uint64_t base,
                                           uint32_t cnt) {
    const uint32_t bulk = bulk_elems<T>(cnt);
#pragma unroll
    for (int s = 0; s < NSUB; ++s) {
        const uint32_t lo = (uint32_t)s * SUB;
        const uint32_t hi = bulk < lo + SUB ? bulk : lo + SUB;
        const uint32_t elems = hi > lo ? hi - lo : 0u;
        mbar_arrive_expect_tx(&bars[s], elems * (uint32_t)sizeof(T));
        if (elems) bulk_load(buf + lo, in + base + lo, elems * (uint32_t)sizeof(T), &bars[s]);
    }
}

// Whole CTA: plain loads for the part of the tile the bulk copies do not cover.
template <typename T, int TILE, int BLOCK>
__device__ __forceinline__ void fill_ragged(T* buf, const T* in, uint64_t base, uint32_t cnt,
                                            uint32_t from) {
    for (uint32_t e = from + threadIdx.x; e < (uint32_t)TILE; e += BLOCK)
        buf[e] = e < cnt ? in[base + e] : T(0);
}

// Non-persistent staging of one tile (used by the allocation-free path and unaligned
// inputs): issues the loads, fills the ragged part, returns the bulk-covered count. Must
// be followed by __syncthreads() before any wait_sub().
template <typename T, int SUB, int NSUB, int BLOCK, bool BULK>
__device__ __forceinline__ uint32_t stage_tile(T* buf, uint64_t* bars, const T* in,
                                               uint64_t base, uint32_t cnt) {
    uint32_t bulk = 0;
    if constexpr (BULK) {
        bulk = bulk_elems<T>(cnt);
        if (threadIdx.x == 0) {
#pragma unroll
            for (int s = 0; s < NSUB; ++s) mbar_init(&bars[s], 1);
            fence_mbar_init();
            issue_tile<T, SUB, NSUB>(buf, bars, in, base, cnt);
        }
    }
    fill_ragged<T, SUB * NSUB, BLOCK>(buf, in, base, cnt, bulk);
    return bulk;
}

// Waits (bounded) until sub-tile s has landed in shared memory.
__device__ __forceinline__ void wait_bar(uint64_t* bar, uint32_t parity, volatile int32_t* err) {
    uint32_t spins = 0;
    while (!mbar_try_wait(bar, parity)) {
        if (++spins > kSpinLimit) {
            *err = 2;
            break;
        }
    }
}
template <bool BULK>
__device__ __forceinline__ void wait_sub(uint64_t* bars, int s, volatile int32_t* err) {
    if constexpr (BULK) wait_bar(&bars[s], 0, err);
}

// Opts a kernel into `bytes` of dynamic shared memory (above the 48 KiB default) on the
// current device. Host side. The attribute belongs to each device's context, so the size
// already set is remembered per device (per kernel instantiation) and the attribute is set
// again on a device that has not seen it, or when a larger size is asked for. A failed
// attempt is not remembered: the next call tries again. On failure the CUDA error stays
// pending for the caller's cudaGetLastError().
constexpr int kSmemOptInDevices = 64;
template <auto Kernel>
inline bool smem_opt_in(size_t bytes) {
    static std::mutex mu;
    static size_t set_bytes[kSmemOptInDevices] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return false;
    if (dev < 0 || dev >= kSmemOptInDevices)  // not remembered: set on every call
        return cudaFuncSetAttribute(Kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)bytes) == cudaSuccess;
    std::lock_guard<std::mutex> g(mu);
    if (set_bytes[dev] >= bytes) return true;
    if (cudaFuncSetAttribute(Kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) !=
        cudaSuccess)
        return false;
    set_bytes[dev] = bytes;
    return true;
}

// Waits until the bulk stores issued by this thread have finished reading shared memory
// (the data may still be on its way to HBM); the CTA may then exit or reuse the buffer.
__device__ __forceinline__ void bulk_wait_read_all() {
    asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}

// One-tile-per-CTA kernels take their tile from an atomic counter (PXB_TILE_CLAIM=1) or
// use blockIdx (0). With a claim counter, a tile's predecessors were all claimed, i.e.
// running, before it, whatever order the hardware dispatches the grid's blocks in; with
// blockIdx the look-back relies on in-order dispatch, and a wait that nonetheless never
// ends gives up after its poll limit with PARALLAX_ERR_DEVICE_SPIN instead of hanging.
#ifndef PXB_TILE_CLAIM
#define PXB_TILE_CLAIM 0
#endif

// Claims the next tile from counters[0]; every thread of the CTA gets it. The CTA must
// call persistent_exit(counters) once at its end, which resets the counters for the next
// launch.
__device__ __forceinline__ uint32_t tile_claim(uint32_t* counters, uint32_t& s_slot) {
    if (threadIdx.x == 0) s_slot = atomicAdd(&counters[0], 1u);
    __syncthreads();
    return s_slot;
}

// Claim / exit counters of a persistent launch: counters[0] hands out tiles,
// counters[1] counts exited CTAs; the last CTA to exit zeroes both for the next launch.
__device__ __forceinline__ void persistent_exit(uint32_t* counters) {
    __threadfence();
    if (atomicAdd(&counters[1], 1u) == gridDim.x - 1) {
        atomicExch(&counters[0], 0u);
        atomicExch(&counters[1], 0u);
    }
}

}  // namespace pxb
