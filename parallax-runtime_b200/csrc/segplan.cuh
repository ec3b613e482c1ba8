// Segment work lists shared by the segmented kernels (segmented.cu, sort.cu).
//
// `offsets` (device, S + 1 entries, CSR) cut the data into segments. The one-CTA planner
// turns segment lengths into a tile work list: item_start[s] = first work item of segment
// s, item_start[S] = total items; a segment of L elements owns ceil(L / tile) items. It
// also writes a caller-chosen value for every empty segment, zeroes a per-segment counter
// array (`seg_zero`, optional), and advances the launch epoch kept in device memory (so a
// replayed CUDA graph gets a fresh epoch every time).
#pragma once

#include "common.cuh"
#include "lookback.cuh"

namespace pxb {

// Largest s with item_start[s] <= item (item_start non-decreasing).
__device__ __forceinline__ uint32_t find_segment(const uint32_t* item_start, uint64_t S,
                                                 uint32_t item) {
    uint64_t lo = 0, hi = S;
    while (hi - lo > 1) {
        const uint64_t mid = (lo + hi) >> 1;
        if (__ldg(&item_start[mid]) <= item) lo = mid;
        else hi = mid;
    }
    return (uint32_t)lo;
}

// Offsets that are not non-decreasing within [0, count] write kErrSegmentOffsets to the
// mapped error word; such segments get no work items, so no kernel touches memory outside
// the caller's buffers.
// counters[2] is the epoch; status (status_cap entries) is cleared when it wraps.
template <typename R, int BLOCK>
__global__ void __launch_bounds__(BLOCK)
k_seg_plan(const uint64_t* __restrict__ offsets, uint64_t S, uint64_t count, uint32_t tile,
           uint32_t* __restrict__ item_start, uint32_t* __restrict__ counters, R* empty_out,
           R empty_value, uint32_t* __restrict__ seg_zero, StatusEntry* status,
           uint64_t status_cap, volatile int32_t* err) {
    __shared__ uint32_t s_warp[BLOCK / 32];
    __shared__ uint32_t s_carry;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) s_carry = 0;
    __syncthreads();
    for (uint64_t base = 0; base < S; base += BLOCK) {
        const uint64_t s = base + tid;
        uint32_t items = 0;
        if (s < S) {
            const uint64_t a = offsets[s], b = offsets[s + 1];
            const bool bad = b < a || b > count;
            if (bad) *err = kErrSegmentOffsets;
            const uint64_t len = bad ? 0 : b - a;
            items = (uint32_t)((len + tile - 1) / tile);
            if (len == 0 && empty_out) empty_out[s] = empty_value;
            if (seg_zero) seg_zero[s] = 0;
        }
        const uint32_t incl = warp_inclusive_scan(items, OpSum());
        if (lane == 31) s_warp[warp] = incl;
        __syncthreads();
        uint32_t woff = 0, total = 0;
#pragma unroll
        for (int w = 0; w < BLOCK / 32; ++w) {
            const uint32_t v = s_warp[w];
            if (w < warp) woff += v;
            total += v;
        }
        if (s < S) item_start[s] = s_carry + woff + incl - items;
        __syncthreads();
        if (tid == 0) s_carry += total;
        __syncthreads();
    }
    if (tid == 0) {
        item_start[S] = s_carry;
        uint32_t e = counters[2] + 1;
        if (e >= (1u << 30)) e = 0;  // wrap: clear the status words below, restart at 1
        counters[2] = e;
    }
    __syncthreads();
    if (counters[2] == 0) {
        for (uint64_t i = tid; i < status_cap; i += BLOCK) status[i].flag = 0;
        __syncthreads();
        if (tid == 0) counters[2] = 1;
    }
}

}  // namespace pxb
