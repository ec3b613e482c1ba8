// Segment work lists shared by the segmented kernels (segmented.cu, sort.cu).
//
// Segments come in one of two forms:
//   CSR         `offsets` (device, S + 1 entries) cut one input array (and the output array
//               at the same offsets) into segments: the segmented ABI entry points;
//   descriptors one SegDesc per segment with its own device addresses: the serving loop's
//               coalesced launches, where every request keeps its operands where they are.
// The one-CTA planner turns segment lengths into a tile work list: item_start[s] = first
// work item of segment s, item_start[S] = total items; a segment of L elements owns
// ceil(L / tile) items. It also writes the results of empty segments (a reduce identity or
// a zero kept count), zeroes a per-segment counter array (optional), and advances the
// launch epoch kept in device memory (so a replayed CUDA graph gets a fresh epoch every
// time).
#pragma once

#include "common.cuh"
#include "lookback.cuh"

namespace pxb {

// One segment of a descriptor-form launch (device-resident table, 32 bytes).
struct SegDesc {
    uint64_t in;   // device address of the segment's input
    uint64_t out;  // device address of its output (scan, copy_if); 0 otherwise
    uint64_t n;    // elements
    uint64_t aux;  // reduce: result address; copy_if: kept-count address (uint64);
                   // sort: address of an n-element temporary
};

// Where segment s lives. CSR: in/out are the arrays' bases, results/counts per-segment
// arrays (aux of a CSR sort is the temporary's base, at the same offsets).
struct SegSrc {
    const uint64_t* offsets;  // CSR form when non-null
    const SegDesc* descs;     // descriptor form otherwise
    uint64_t in, out, aux;    // CSR bases (addresses)
    uint32_t aux_stride;      // CSR: bytes per segment of the aux array (result / count)
    uint32_t elem;            // element bytes

    __device__ __forceinline__ uint64_t begin(uint64_t s) const {
        return offsets ? __ldg(&offsets[s]) : 0;
    }
    __device__ __forceinline__ uint64_t len(uint64_t s) const {
        return offsets ? __ldg(&offsets[s + 1]) - __ldg(&offsets[s]) : descs[s].n;
    }
    __device__ __forceinline__ uint64_t in_addr(uint64_t s) const {
        return offsets ? in + begin(s) * elem : descs[s].in;
    }
    __device__ __forceinline__ uint64_t out_addr(uint64_t s) const {
        return offsets ? out + begin(s) * elem : descs[s].out;
    }
    // reduce result / copy_if count slot, or the sort temporary of the segment
    __device__ __forceinline__ uint64_t aux_addr(uint64_t s) const {
        if (!offsets) return descs[s].aux;
        return aux_stride ? aux + s * aux_stride : aux + begin(s) * elem;
    }
};

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

// Inverse of the work list: item_seg[i] = the segment of work item i, so a kernel finds
// its segment with one load instead of a binary search. One thread per segment writes
// that segment's items (grid-stride over segments). Work lists of at most kInlineItems
// items get it from the planner itself (`item_seg` argument) instead.
constexpr uint64_t kInlineItems = 16384;
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK)
k_seg_map(const uint32_t* __restrict__ item_start, uint64_t S, uint32_t* __restrict__ item_seg) {
    for (uint64_t s = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; s < S;
         s += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t a = item_start[s], b = item_start[s + 1];
        for (uint32_t i = a; i < b; ++i) item_seg[i] = (uint32_t)s;
    }
}
inline unsigned seg_map_grid(uint64_t S) {  // for BLOCK = 256
    const uint64_t g = (S + 255) / 256;
    return (unsigned)(g < 1024 ? (g ? g : 1) : 1024);
}

// What the planner writes for an empty segment.
enum class SegEmpty : int { NONE = 0, ZERO_RESULT = 1, ZERO_COUNT = 2 };

// counters[2] is the epoch; status (status_cap entries) is cleared when it wraps.
// CSR offsets that are not non-decreasing within [0, count] write kErrSegmentOffsets to the
// mapped error word; such segments get no work items, so no kernel touches memory outside
// the caller's buffers.
// The planner's work, by one CTA of BLOCK threads (k_seg_plan; planners that go on to write
// more of the work list call it first).
template <int BLOCK>
__device__ __forceinline__ void seg_plan_block(SegSrc src, uint64_t S, uint64_t count,
                                               uint32_t tile, uint32_t* item_start,
                                               uint32_t* counters, SegEmpty empty,
                                               uint32_t* seg_zero, StatusEntry* status,
                                               uint64_t status_cap, volatile int32_t* err,
                                               uint32_t* item_seg) {
    // Each thread takes kPer consecutive segments of a chunk and issues all their length
    // loads before using any, so a chunk of BLOCK * kPer segments costs about one memory
    // round trip (one segment per thread per chunk made S = 4096 sixteen dependent rounds).
    constexpr int kPer = 16;
    __shared__ uint32_t s_warp[BLOCK / 32];
    __shared__ uint32_t s_carry;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) s_carry = 0;
    __syncthreads();
    for (uint64_t base = 0; base < S; base += (uint64_t)BLOCK * kPer) {
        const uint64_t s0 = base + (uint64_t)tid * kPer;
        uint64_t len[kPer];
        if (src.offsets) {
            uint64_t o[kPer + 1];
#pragma unroll
            for (int j = 0; j <= kPer; ++j) o[j] = s0 + j <= S ? src.offsets[s0 + j] : 0;
#pragma unroll
            for (int j = 0; j < kPer; ++j) {
                const bool bad = o[j + 1] < o[j] || o[j + 1] > count;
                if (s0 + j < S && bad) *err = kErrSegmentOffsets;
                len[j] = s0 + j < S && !bad ? o[j + 1] - o[j] : 0;
            }
        } else {
#pragma unroll
            for (int j = 0; j < kPer; ++j) len[j] = s0 + j < S ? src.descs[s0 + j].n : 0;
        }
        uint32_t items[kPer];
        uint32_t mine = 0;
#pragma unroll
        for (int j = 0; j < kPer; ++j) {
            items[j] = (uint32_t)((len[j] + tile - 1) / tile);
            mine += items[j];
            if (s0 + j >= S) continue;
            if (len[j] == 0 && empty != SegEmpty::NONE) {
                void* slot = reinterpret_cast<void*>(src.aux_addr(s0 + j));
                if (empty == SegEmpty::ZERO_COUNT) *static_cast<uint64_t*>(slot) = 0;
                else if (src.elem == 8) *static_cast<uint64_t*>(slot) = 0;  // +0.0 / 0
                else *static_cast<uint32_t*>(slot) = 0;
            }
            if (seg_zero) seg_zero[s0 + j] = 0;
        }
        const uint32_t incl = warp_inclusive_scan(mine, OpSum());
        if (lane == 31) s_warp[warp] = incl;
        __syncthreads();
        uint32_t woff = 0, total = 0;
#pragma unroll
        for (int w = 0; w < BLOCK / 32; ++w) {
            const uint32_t v = s_warp[w];
            if (w < warp) woff += v;
            total += v;
        }
        uint32_t first = s_carry + woff + incl - mine;
#pragma unroll
        for (int j = 0; j < kPer; ++j) {
            if (s0 + j >= S) break;
            item_start[s0 + j] = first;
            if (item_seg)  // small work lists: the inverse map too (saves a launch)
                for (uint32_t i = 0; i < items[j]; ++i) item_seg[first + i] = (uint32_t)(s0 + j);
            first += items[j];
        }
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
        for (uint64_t i = tid; i < status_cap; i += BLOCK) status[i] = StatusEntry{0u, 0u, 0u, 0u};
        __syncthreads();
        if (tid == 0) counters[2] = 1;
    }
}

template <int BLOCK>
__global__ void __launch_bounds__(BLOCK)
k_seg_plan(SegSrc src, uint64_t S, uint64_t count, uint32_t tile,
           uint32_t* __restrict__ item_start, uint32_t* __restrict__ counters, SegEmpty empty,
           uint32_t* __restrict__ seg_zero, StatusEntry* status, uint64_t status_cap,
           volatile int32_t* err, uint32_t* __restrict__ item_seg) {
    seg_plan_block<BLOCK>(src, S, count, tile, item_start, counters, empty, seg_zero, status,
                          status_cap, err, item_seg);
}

struct Workspace;

// Segmented radix sort (kernels/radix.cu): each of the S segments of `src` sorted in place,
// one histogram launch and one launch per digit pass for all of them; by_key: 8-byte
// (key << 32 | value) records sorted stably by key (four passes). CSR segments need
// src.aux unset (the temporary comes from the workspace), descriptors carry their own.
// `graph`: captured once per argument set as a CUDA graph and replayed.
bool launch_segmented_radix_sort(Workspace& ws, DType t, const SegSrc& src, uint64_t count,
                                 uint64_t S, bool by_key, bool graph);
// Keys per tile (work item) of the segmented radix sort.
uint64_t segmented_radix_tile(DType t);

}  // namespace pxb
