// Segmented primitives: thousands of uneven segments in ONE persistent launch.
//
// No reference counterpart (the reference dispatches one primitive call per array,
// src/kernel/kernel_launcher.cpp); this is the batching path of the B200 design. Per
// segment, each primitive computes exactly what the reference's primitive computes for one
// array: reduce (sum / max / min), inclusive and exclusive scan, copy_if / remove_if,
// stable partition, unique (kernel_launcher.cpp:819-1791).
//
// Segments are either CSR (`offsets`, device, num_segments + 1 entries, cut one input
// array and the output array at the same offsets) or descriptors (one device-resident
// SegDesc per segment with its own addresses, used by the serving loop to coalesce
// requests without moving their operands). A one-CTA planner kernel turns the segment
// lengths into a tile work list (item_start[s] = first work item of segment s; a segment of
// L elements has ceil(L / tile) items) and writes the results of empty segments; the
// persistent kernel's CTAs then claim work items from an atomic counter in order and
// process one tile each. A work item's descriptor (segment, tile index, addresses) is
// precomputed, and thread 0 claims and describes the next item while the current tile's
// results are being stored (a reduce tile: while it is being read), so the claim's round
// trip and the descriptor load overlap the work of the previous tile.
//
// A tile is staged in shared memory with 16-byte vector loads (striped: consecutive
// threads read consecutive vectors), at the segment's own 16-byte phase: element e of the
// tile sits at slot e + mis, mis = the start's misalignment in elements, so every vector
// inside the tile is one aligned load and only the (at most two) ragged vectors at its ends
// are read element by element. Each thread then owns a row of VPT consecutive vectors; VPT
// is odd, so the 16-byte row reads of a warp hit every bank once. Tiles hold
// BLOCK x VPT vectors minus one (room for the phase shift).
//   reduce     per-tile sum (max, min, or predicate count) -> per-item partial; the last
//              tile of a segment to finish (per-segment ticket) folds the partials in item
//              order (deterministic)
//   scan       row scans + warp shuffles + decoupled look-back that stops at the segment's
//              first tile; results written back into the staged rows and stored with
//              16-byte stores when the output has the input's phase
//   select     predicate (or adjacent-difference for unique) flags, one ballot per 32
//              consecutive elements (warp-strided walk of the staged tile), look-back on kept
//              counts within the segment, each ballot's kept run stored from the tile
//   partition  select's ranks for both runs: kept elements to the front of the segment's
//              output, rejected ones after the segment's kept total (a count pass first)
// The tile shape (BLOCK x VPT) is picked per (operation, element type, log2 of the mean
// segment length) by timing the candidates on the first call (the autotuner); every CSR
// launch sequence is captured once per argument set as a CUDA graph and replayed; the
// look-back epoch lives in device memory and is advanced by the planner, so a replay never
// reads status words of an earlier replay.
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <limits>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <type_traits>

#include "../lookback.cuh"
#include "../runtime.hpp"
#include "../segplan.cuh"
#include "../tiles.cuh"

namespace pxb {
namespace {

// Tile shapes the autotuner chooses from: (threads per CTA, 16-byte vectors per thread).
struct TileShape {
    int block, vpt;
};
constexpr TileShape kShapes[] = {{256, 3}, {256, 7}, {512, 7}};
constexpr int kNumShapes = 3;

enum SegOp : int { SEG_REDUCE = 0, SEG_SCAN = 1, SEG_SELECT = 2, SEG_PARTITION = 3 };
// reduce flavours
enum SegRed : int { RED_SUM = 0, RED_MAX = 1, RED_MIN = 2, RED_COUNT = 3 };

template <typename T, int BLOCK, int VPT>
struct SegShape {
    static constexpr int V = 16 / sizeof(T);
    static constexpr int ITEMS = VPT * V;            // elements per thread row
    static constexpr int SLOTS = BLOCK * ITEMS;      // staged slots
    static constexpr int TILE = SLOTS - V;           // tile elements (room for the phase)
    static constexpr size_t SMEM = SLOTS * sizeof(T);
};

// Device buffers of one segmented launch (the workspace's segment and status buffers).
// Everything a CTA needs to find its tile, precomputed per work item (48 bytes, read with
// three 16-byte loads), so claiming an item costs one load after the claim, not a chain of
// dependent loads (item -> segment -> segment bounds -> addresses).
struct __align__(16) ItemDesc {
    uint32_t seg, first_item, seg_items, k;  // segment, its first item and item count, k = item - first
    uint64_t len, in, out, aux;              // segment length and addresses
};
static_assert(sizeof(ItemDesc) == 48, "item descriptor layout");

struct SegBuffers {
    uint32_t* item_start;  // num_segments + 1
    ItemDesc* items;       // one per work item
    uint64_t* partials;    // one per work item
    StatusEntry* status;   // one per work item (a buffer of its own)
    uint64_t status_cap;   // entries in that buffer
    uint32_t* counters;    // [0] claim, [1] exit, [2] epoch, [3] error
};

// Predicate of the segmented select / partition / count: comparisons, x % m == r on
// integers (32-bit element types by the invariant-divisor remainder), nonzero.
template <typename T>
struct SegPred {
    PredKind kind;
    bool negate;
    T c, m, r;
    FastMod32 fm;
    __device__ __forceinline__ bool operator()(T x) const {
        bool v;
        switch (kind) {
            case PredKind::GT: v = x > c; break;
            case PredKind::GE: v = x >= c; break;
            case PredKind::LT: v = x < c; break;
            case PredKind::LE: v = x <= c; break;
            case PredKind::EQ: v = x == c; break;
            case PredKind::NE: v = x != c; break;
            case PredKind::NONZERO: v = x != T(0); break;
            case PredKind::MOD:
                if constexpr (std::is_integral<T>::value && sizeof(T) == 4) {
                    v = fm.eq(x, r);
                } else if constexpr (std::is_integral<T>::value) {
                    v = (std::is_signed<T>::value && m == T(-1)) ? r == T(0) : x % m == r;
                } else {
                    v = false;
                }
                break;
            default: v = false; break;
        }
        return v != negate;
    }
};

template <typename T> struct SegAcc { using type = typename SumAcc<T>::type; };
// Type of a row's running sum in the scan: fp32 rows sum in fp32 (at most 28 terms), and
// rows, warps and tiles are carried in fp64; integers wrap in their unsigned type.
template <typename T> struct SegRow { using type = typename SumAcc<T>::type; };
template <> struct SegRow<float> { using type = float; };

// Per-launch parameters.
template <typename T>
struct SegArgs {
    SegSrc src;
    uint64_t S;
    T init;            // exclusive scan init
    bool inclusive;    // scan flavour
    bool unique;       // select: adjacent-difference flags instead of the predicate
    int red;           // reduce flavour (SegRed)
    SegPred<T> pred;
};

// Writes the descriptor of every work item (one thread per item, grid-stride): the item's
// segment is found by binary search over the planner's item_start.
__global__ void __launch_bounds__(256)
k_item_descs(SegSrc src, uint64_t S, const uint32_t* __restrict__ item_start,
             ItemDesc* __restrict__ items) {
    const uint32_t total = item_start[S];
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += gridDim.x * blockDim.x) {
        const uint32_t s = find_segment(item_start, S, i);
        ItemDesc d;
        d.seg = s;
        d.first_item = item_start[s];
        d.seg_items = item_start[s + 1] - d.first_item;
        d.k = i - d.first_item;
        d.len = src.len(s);
        d.in = src.in_addr(s);
        d.out = src.out_addr(s);
        d.aux = src.aux_addr(s);
        items[i] = d;
    }
}

// The planner and k_item_descs in one launch, for work lists of at most kPlanItemsMax
// items (one launch less per call: a batch of small requests costs its host thread a
// launch, not the device time). item_start is read back with plain loads: this CTA wrote it.
constexpr uint64_t kPlanItemsMax = 8192;
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK)
k_seg_plan_items(SegSrc src, uint64_t S, uint64_t count, uint32_t tile, uint32_t* item_start,
                 uint32_t* counters, SegEmpty empty, uint32_t* seg_zero, StatusEntry* status,
                 uint64_t status_cap, volatile int32_t* err, ItemDesc* __restrict__ items) {
    seg_plan_block<BLOCK>(src, S, count, tile, item_start, counters, empty, seg_zero, status,
                          status_cap, err, nullptr);
    __syncthreads();
    const uint32_t total = item_start[S];
    for (uint32_t i = threadIdx.x; i < total; i += BLOCK) {
        uint64_t lo = 0, hi = S;  // largest s with item_start[s] <= i
        while (hi - lo > 1) {
            const uint64_t mid = (lo + hi) >> 1;
            if (item_start[mid] <= i) lo = mid;
            else hi = mid;
        }
        ItemDesc d;
        d.seg = (uint32_t)lo;
        d.first_item = item_start[lo];
        d.seg_items = item_start[lo + 1] - d.first_item;
        d.k = i - d.first_item;
        d.len = src.len(lo);
        d.in = src.in_addr(lo);
        d.out = src.out_addr(lo);
        d.aux = src.aux_addr(lo);
        items[i] = d;
    }
}

__device__ __forceinline__ ItemDesc load_desc(const ItemDesc* items, uint32_t i) {
    const uint4* p = reinterpret_cast<const uint4*>(items + i);
    uint4 w[3];
#pragma unroll
    for (int q = 0; q < 3; ++q) w[q] = __ldg(p + q);
    ItemDesc d;
    memcpy(&d, w, sizeof d);
    return d;
}

// Stages tile elements [begin, begin + len) of `in` so that slot e + mis holds element e
// (mis = the misalignment of in + begin in elements); other slots get `pad`. Vectors
// entirely inside the tile are single 16-byte loads; the ragged ones element by element.
template <typename T, int BLOCK, int VPT>
__device__ __forceinline__ void stage(T* sm, const T* in, uint64_t begin, uint32_t len,
                                      uint32_t mis, T pad) {
    using Sh = SegShape<T, BLOCK, VPT>;
    constexpr int V = Sh::V;
    const T* base = in + begin - mis;  // 16-byte aligned when in is element-aligned
#pragma unroll
    for (int k = 0; k < VPT; ++k) {
        const int j = k * BLOCK + threadIdx.x;
        const int e0 = j * V - (int)mis;  // tile index of the vector's first slot
        uint4 v;
        if (e0 >= 0 && e0 + V <= (int)len) {
            v = *reinterpret_cast<const uint4*>(base + j * V);
        } else {
            T* e = reinterpret_cast<T*>(&v);
#pragma unroll
            for (int q = 0; q < V; ++q) {
                const int i = e0 + q;
                e[q] = (i >= 0 && i < (int)len) ? base[j * V + q] : pad;
            }
        }
        *reinterpret_cast<uint4*>(sm + j * V) = v;
    }
}

// Writes slots [mis, mis + len) of sm to out[begin ...]: 16-byte stores when the output
// start has the same phase as the staged tile, element stores otherwise.
template <typename T, int BLOCK, int VPT>
__device__ __forceinline__ void unstage(const T* sm, T* out, uint64_t begin, uint32_t len,
                                        uint32_t mis) {
    using Sh = SegShape<T, BLOCK, VPT>;
    constexpr int V = Sh::V;
    const uint32_t omis = (uint32_t)((reinterpret_cast<uintptr_t>(out + begin) % 16) / sizeof(T));
    if (omis == mis && reinterpret_cast<uintptr_t>(out) % sizeof(T) == 0) {
        T* base = out + begin - mis;
#pragma unroll
        for (int k = 0; k < VPT; ++k) {
            const int j = k * BLOCK + threadIdx.x;
            const int e0 = j * V - (int)mis;
            if (e0 >= 0 && e0 + V <= (int)len) {
                *reinterpret_cast<uint4*>(base + j * V) = *reinterpret_cast<const uint4*>(sm + j * V);
            } else {
#pragma unroll
                for (int q = 0; q < V; ++q) {
                    const int i = e0 + q;
                    if (i >= 0 && i < (int)len) base[j * V + q] = sm[j * V + q];
                }
            }
        }
    } else {
        for (uint32_t e = threadIdx.x; e < len; e += BLOCK) out[begin + e] = sm[e + mis];
    }
}

template <int BLOCK, typename A, typename Op>
__device__ __forceinline__ A block_fold(A v, A* red, Op op) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    v = warp_reduce(v, op);
    if (lane == 0) red[warp] = v;
    __syncthreads();
    A t = red[0];
#pragma unroll
    for (int w = 1; w < BLOCK / 32; ++w) t = op(t, red[w]);
    __syncthreads();
    return t;
}

template <typename T>
__device__ __forceinline__ T red_identity(int red) {
    if (red == RED_MAX)
        return std::numeric_limits<T>::has_infinity ? -std::numeric_limits<T>::infinity()
                                                    : std::numeric_limits<T>::lowest();
    if (red == RED_MIN)
        return std::numeric_limits<T>::has_infinity ? std::numeric_limits<T>::infinity()
                                                    : std::numeric_limits<T>::max();
    return T(0);
}

// Rank scan of a row's kept-flag count over the CTA: this row's kept elements start at
// woff + tex within the tile; returns the tile's kept total.
template <int BLOCK>
__device__ __forceinline__ uint32_t tile_ranks(uint32_t cnt, uint32_t* wcnt, uint32_t* start) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t incl = warp_inclusive_scan(cnt, OpSum());
    if (lane == 31) wcnt[warp] = incl;
    __syncthreads();
    uint32_t woff = 0, tot = 0;
#pragma unroll
    for (int w = 0; w < BLOCK / 32; ++w) {
        const uint32_t v = wcnt[w];
        if (w < warp) woff += v;
        tot += v;
    }
    *start = woff + incl - cnt;
    return tot;
}

// Select / partition tiles walked warp-strided with one ballot per 32 elements
// (PXB_SEG_STRIDED=1) instead of thread rows packed in shared memory (0). Measured on the
// 4096-segment lognormal workload (122 M elements, x > 0.5 / x > 0): copy_if fp32 0.480 ms
// strided against 0.550 ms in rows, int32 0.497 against 0.566 ms. (The same walk made the
// plain compaction kernels slower - copy_if 0.56 against 0.40 ms at 2^28 - whose rows read
// their 112 KiB tiles with 16-byte loads and store packed runs; it is not used there.)
#ifndef PXB_SEG_STRIDED
#define PXB_SEG_STRIDED 1
#endif

__device__ __forceinline__ uint32_t lane_mask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Second pass of a segmented reduce (and of the partition's count pass): one warp per
// segment of more than one work item folds the items' partials in item order (lane-strided,
// then the warp's tree) and writes the segment's result; one-item segments were written by
// their item. A pass of its own instead of a last-arriving-item ticket keeps the fence and
// the atomic off every item's path.
template <typename T>
__global__ void __launch_bounds__(256)
k_seg_fold(SegBuffers b, uint64_t S, int red) {
    using A = typename SegAcc<T>::type;
    const uint64_t s = ((uint64_t)blockIdx.x * 256 + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (s >= S) return;
    const uint32_t first = b.item_start[s], n = b.item_start[s + 1] - first;
    if (n < 2) return;
    const uint64_t aux = b.items[first].aux;
    if (red == RED_MAX || red == RED_MIN) {
        T m = red_identity<T>(red);
        for (uint32_t i = lane; i < n; i += 32) {
            const T v = get_val<T>(&b.partials[first + i]);
            m = red == RED_MAX ? OpMax()(m, v) : OpMin()(m, v);
        }
        m = red == RED_MAX ? warp_reduce(m, OpMax()) : warp_reduce(m, OpMin());
        if (lane == 0) *reinterpret_cast<T*>(aux) = m;
    } else {
        A f = A(0);
        for (uint32_t i = lane; i < n; i += 32) f = f + get_val<A>(&b.partials[first + i]);
        f = warp_reduce(f, OpSum());
        if (lane == 0) {
            if (red == RED_COUNT) *reinterpret_cast<uint64_t*>(aux) = (uint64_t)f;
            else *reinterpret_cast<T*>(aux) = (T)f;
        }
    }
}

// ---- the persistent kernel -------------------------------------------------------------------------
template <typename T, int BLOCK, int VPT, int OP>
__global__ void __launch_bounds__(BLOCK)
k_segmented(SegArgs<T> a, SegBuffers b, volatile int32_t* err) {
    using Sh = SegShape<T, BLOCK, VPT>;
    using A = typename SegAcc<T>::type;
    constexpr int V = Sh::V;
    constexpr int ITEMS = Sh::ITEMS;
    constexpr int TILE = Sh::TILE;
    constexpr int WARPS = BLOCK / 32;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* sm = reinterpret_cast<T*>(smem_raw);
    __shared__ A red[WARPS + 1];
    __shared__ uint64_t red64[WARPS + 1];
    __shared__ T redT[WARPS + 1];
    __shared__ int first[WARPS];
    __shared__ uint32_t wcnt[WARPS];
    __shared__ ItemDesc s_it;
    __shared__ uint32_t s_item;
    __shared__ T s_prev;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t total = b.item_start[a.S];
    TileStatus<A> ts;
    ts.e = b.status;
    ts.epoch = b.counters[2];
    ts.err = err;
    TileStatus<uint64_t> tsk;
    tsk.e = b.status;
    tsk.epoch = b.counters[2];
    tsk.err = err;

    // Thread 0 claims the next item and loads its descriptor while the current tile is still
    // in progress, so the claim's round trip and the dependent descriptor load overlap work.
    // A look-back tile claims its successor only once its own inclusive prefix is published
    // (before its stores): a claimed item that waits behind a tile still in its look-back
    // would hold up every later tile's look-back for a whole tile. Reduce tiles never wait,
    // and claim at their start. Claims are made in order and a CTA works on its claims in
    // order, so the lowest unfinished item is always being worked on: every look-back ends.
    uint32_t c_next = 0;
    ItemDesc d_next;
    if (tid == 0) {
        c_next = atomicAdd(&b.counters[0], 1u);
        if (c_next < total) d_next = load_desc(b.items, c_next);
    }
    auto claim_next = [&]() {
        if (tid == 0) c_next = atomicAdd(&b.counters[0], 1u);
    };
    auto describe_next = [&]() {
        if (tid == 0 && c_next < total) d_next = load_desc(b.items, c_next);
    };
    for (;;) {
        if (tid == 0) {
            s_item = c_next;
            if (c_next < total) s_it = d_next;
        }
        __syncthreads();
        const ItemDesc it = s_it;
        const uint32_t item = s_item;
        if (item >= total) break;
        const uint32_t k = it.k;  // tile index within the segment
        const uint64_t begin = (uint64_t)k * TILE;   // within the segment
        const uint32_t len = (uint32_t)min((uint64_t)TILE, it.len - begin);
        const T* in = reinterpret_cast<const T*>(it.in);
        T* out = reinterpret_cast<T*>(it.out);
        const uint32_t mis = (reinterpret_cast<uintptr_t>(in) % sizeof(T)) ? 0u
            : (uint32_t)((reinterpret_cast<uintptr_t>(in + begin) % 16) / sizeof(T));
        const bool vec_ok = reinterpret_cast<uintptr_t>(in) % sizeof(T) == 0;

        if constexpr (OP == SEG_REDUCE) {
            claim_next();
            describe_next();
            // straight from global memory: each thread first issues all of its VPT vector
            // loads (streaming, no L1 allocation), then folds them; sums and counts
            // accumulate in A, max / min in T
            const bool mm = a.red == RED_MAX || a.red == RED_MIN;
            A acc = A(0);
            T accm = red_identity<T>(a.red);
            const T* base = in + begin - mis;
            uint4 v[VPT];
#pragma unroll
            for (int q = 0; q < VPT; ++q) {
                const int j = q * BLOCK + tid;
                const int e0 = j * V - (int)mis;
                v[q] = vec_ok && e0 >= 0 && e0 + V <= (int)len
                           ? ldg_stream16(base + j * V)
                           : make_uint4(0u, 0u, 0u, 0u);
            }
            auto fold = [&](auto red_c) {
                constexpr int R = decltype(red_c)::value;
#pragma unroll
                for (int q = 0; q < VPT; ++q) {
                    const int e0 = (q * BLOCK + tid) * V - (int)mis;
                    const bool full = vec_ok && e0 >= 0 && e0 + V <= (int)len;
                    T x[V];
                    memcpy(x, &v[q], 16);
#pragma unroll
                    for (int e = 0; e < V; ++e) {
                        const int i = e0 + e;
                        const bool in_tile = i >= 0 && i < (int)len;
                        if (!full && in_tile) x[e] = in[begin + i];  // the ragged ends
                        if (full || in_tile) {
                            if constexpr (R == RED_SUM) acc = acc + (A)x[e];
                            else if constexpr (R == RED_COUNT) acc = acc + (A)(a.pred(x[e]) ? 1 : 0);
                            else if constexpr (R == RED_MAX) accm = OpMax()(accm, x[e]);
                            else accm = OpMin()(accm, x[e]);
                        }
                    }
                }
            };
            switch (a.red) {
                case RED_SUM: fold(std::integral_constant<int, RED_SUM>()); break;
                case RED_COUNT: fold(std::integral_constant<int, RED_COUNT>()); break;
                case RED_MAX: fold(std::integral_constant<int, RED_MAX>()); break;
                default: fold(std::integral_constant<int, RED_MIN>()); break;
            }
            const bool count = a.red == RED_COUNT;
            A tot = A(0);
            T totm = accm;
            if (a.red == RED_MAX) totm = block_fold<BLOCK>(accm, redT, OpMax());
            else if (a.red == RED_MIN) totm = block_fold<BLOCK>(accm, redT, OpMin());
            else tot = block_fold<BLOCK>(acc, red, OpSum());
            auto write = [&](A sum, T m) {
                if (count) *reinterpret_cast<uint64_t*>(it.aux) = (uint64_t)sum;
                else *reinterpret_cast<T*>(it.aux) = mm ? m : (T)sum;
            };
            // A one-item segment's result is final; otherwise the item leaves its partial
            // for k_seg_fold (no fence, ticket or extra barrier on the item's path: the next
            // item's loads follow at once). block_fold's closing barrier has ordered every
            // read of s_it and of the fold scratch before the next claim overwrites them.
            if (tid == 0) {
                if (it.seg_items == 1) write(tot, totm);
                else if (mm) put_val(&b.partials[item], totm);
                else put_val(&b.partials[item], tot);
            }
        } else {
            if (vec_ok) {
                stage<T, BLOCK, VPT>(sm, in, begin, len, mis, T(0));
            } else {  // element-misaligned pointer: element loads only
                for (int s = tid; s < Sh::SLOTS; s += BLOCK) sm[s] = s < (int)len ? in[begin + s] : T(0);
            }
            if (OP == SEG_SELECT && a.unique && tid == 0)
                s_prev = begin > 0 ? in[begin - 1] : T(0);
            __syncthreads();
            // this thread's row: slots [tid * ITEMS, +ITEMS) = tile indices from r0
            [[maybe_unused]] const int r0 = tid * ITEMS - (int)mis;
            T x[ITEMS];
            {
                const uint4* row = reinterpret_cast<const uint4*>(sm + tid * ITEMS);
#pragma unroll
                for (int v = 0; v < VPT; ++v) {
                    const uint4 q = row[v];
                    memcpy(&x[v * V], &q, 16);
                }
            }
            if constexpr (OP == SEG_SCAN) {
                using L = typename SegRow<T>::type;
                L p[ITEMS];
                p[0] = (L)x[0];
#pragma unroll
                for (int j = 1; j < ITEMS; ++j) p[j] = p[j - 1] + (L)x[j];
                const A incl = warp_inclusive_scan((A)p[ITEMS - 1], OpSum());
                A tex = shfl_up(incl, 1);
                if (lane == 0) tex = A(0);
                if (lane == 31) red[warp] = incl;
                __syncthreads();
                A woff = A(0), agg = A(0);
#pragma unroll
                for (int w = 0; w < WARPS; ++w) {
                    if (w < warp) woff = woff + red[w];
                    agg = agg + red[w];
                }
                __syncthreads();
                const A prefix =
                    lookback_cta<A, BLOCK>(ts, item, agg, red, first, it.first_item);
                claim_next();
                const A tb = (A)a.init + ((prefix + woff) + tex);
                uint4* row = reinterpret_cast<uint4*>(sm + tid * ITEMS);
#pragma unroll
                for (int v = 0; v < VPT; ++v) {
                    T o[V];
#pragma unroll
                    for (int q = 0; q < V; ++q) {
                        const int j = v * V + q;
                        o[q] = a.inclusive ? (T)(tb + (A)p[j]) : (T)(j == 0 ? tb : tb + (A)p[j - 1]);
                    }
                    uint4 w;
                    memcpy(&w, o, 16);
                    row[v] = w;
                }
                __syncthreads();
                if (reinterpret_cast<uintptr_t>(out) % sizeof(T) == 0 && vec_ok)
                    unstage<T, BLOCK, VPT>(sm, out, begin, len, mis);
                else
                    for (uint32_t e = tid; e < len; e += BLOCK) out[begin + e] = sm[e + mis];
                describe_next();
                __syncthreads();
            } else if constexpr (PXB_SEG_STRIDED) {  // SEG_SELECT / SEG_PARTITION, strided
                // Warp w walks its slots [w * 32 * ITEMS, + 32 * ITEMS) 32 at a time: lane l
                // holds slot w0 + 32 j + l (element slot - mis). One ballot per j ranks the
                // kept lanes; each j's kept (and rejected) elements are one contiguous output
                // run, stored straight from the staged tile.
                const uint32_t lt = lane_mask_lt();
                const int w0 = warp * 32 * ITEMS;
                T xs[ITEMS];
#pragma unroll
                for (int j = 0; j < ITEMS; ++j) xs[j] = sm[w0 + 32 * j + lane];
                uint32_t mine = 0;  // lane j: kept lanes of item j
#pragma unroll
                for (int j = 0; j < ITEMS; ++j) {
                    const int i = w0 + 32 * j + lane - (int)mis;  // element index in the tile
                    bool keep;
                    if (OP == SEG_SELECT && a.unique) {
                        const T up = shfl_up(xs[j], 1);
                        const T l31 = j > 0 ? shfl_idx(xs[j > 0 ? j - 1 : 0], 31)
                                            : (w0 > 0 ? sm[w0 - 1] : s_prev);
                        const T prev = i == 0 ? s_prev : lane > 0 ? up : l31;
                        keep = (begin == 0 && i == 0) || !(xs[j] == prev);
                    } else {
                        keep = a.pred(xs[j]);
                    }
                    const uint32_t m = __ballot_sync(0xffffffffu, keep && i >= 0 && i < (int)len);
                    if (lane == j) mine = m;
                }
                uint32_t kstart;  // lane j: kept elements of the tile before item j of this warp
                const uint32_t kept = tile_ranks<BLOCK>((uint32_t)__popc(mine), wcnt, &kstart);
                const uint64_t prefix =
                    lookback_cta<uint64_t, BLOCK>(tsk, item, (uint64_t)kept, red64, first,
                                                  it.first_item);
                claim_next();
                uint64_t rej_base = 0;  // partition: position of the tile's first rejected one
                if constexpr (OP == SEG_PARTITION)
                    rej_base = *reinterpret_cast<const uint64_t*>(it.aux) + (begin - prefix);
#pragma unroll 4
                for (int j = 0; j < ITEMS; ++j) {
                    const uint32_t m = shfl_idx(mine, j);
                    const uint32_t ks = shfl_idx(kstart, j);
                    const int i = w0 + 32 * j + lane - (int)mis;
                    if (i < 0 || i >= (int)len) continue;
                    const uint32_t kept_before = ks + (uint32_t)__popc(m & lt);  // in the tile
                    uint64_t dst;
                    if (m >> lane & 1u) dst = prefix + kept_before;
                    else if constexpr (OP == SEG_PARTITION) dst = rej_base + ((uint32_t)i - kept_before);
                    else continue;
                    if (dst < it.len) out[dst] = sm[w0 + 32 * j + lane];
                    else *err = 3;
                }
                if (OP == SEG_SELECT && tid == 0 && k == it.seg_items - 1)
                    *reinterpret_cast<uint64_t*>(it.aux) = prefix + kept;
                describe_next();
                __syncthreads();
            } else {  // SEG_SELECT / SEG_PARTITION
                uint32_t f = 0;
#pragma unroll
                for (int j = 0; j < ITEMS; ++j) {
                    const int i = r0 + j;
                    bool keep;
                    if (OP == SEG_SELECT && a.unique) {
                        const T prev = i == 0 ? s_prev : j > 0 ? x[j - 1] : sm[tid * ITEMS - 1];
                        keep = (begin == 0 && i == 0) || !(x[j] == prev);
                    } else {
                        keep = a.pred(x[j]);
                    }
                    if (i >= 0 && i < (int)len && keep) f |= 1u << j;
                }
                uint32_t kstart;
                const uint32_t kept = tile_ranks<BLOCK>(__popc(f), wcnt, &kstart);
                const uint64_t prefix =
                    lookback_cta<uint64_t, BLOCK>(tsk, item, (uint64_t)kept, red64, first,
                                                  it.first_item);
                claim_next();
                // Output warp by warp: warp w's rows are the staged slots [w * 32 * ITEMS,
                // + 32 * ITEMS), whose kept elements form one contiguous output run (and, for
                // partition, whose rejected ones form another), so each warp packs its own
                // slots in place and stores its runs with no CTA-wide barrier.
                T* const wsm = sm + warp * 32 * ITEMS;
                {  // the row again, from shared memory (fewer registers live across the look-back)
                    const uint4* row = reinterpret_cast<const uint4*>(sm + tid * ITEMS);
#pragma unroll
                    for (int v = 0; v < VPT; ++v) {
                        const uint4 q = row[v];
                        memcpy(&x[v * V], &q, 16);
                    }
                }
                __syncwarp();  // every row of the warp is in registers before it is overwritten
                const uint32_t wex = shfl_idx(kstart, 0);                      // kept before the warp
                const uint32_t wk = shfl_idx(kstart + (uint32_t)__popc(f), 31) - wex;
                uint32_t rk = kstart - wex;
                if constexpr (OP == SEG_SELECT) {
#pragma unroll
                    for (int j = 0; j < ITEMS; ++j)
                        if (f >> j & 1u) wsm[rk++] = x[j];
                    __syncwarp();
                    for (uint32_t i = lane; i < wk; i += 32) {
                        if (prefix + wex + i < it.len) out[prefix + wex + i] = wsm[i];
                        else *err = 3;
                    }
                    if (tid == 0 && k == it.seg_items - 1)
                        *reinterpret_cast<uint64_t*>(it.aux) = prefix + kept;
                } else {
                    // rejected elements of the warp follow its kept run in its slots
                    uint32_t valid = 0;
#pragma unroll
                    for (int j = 0; j < ITEMS; ++j) valid += (r0 + j >= 0 && r0 + j < (int)len);
                    const uint32_t rej = valid - __popc(f);
                    const uint32_t rincl = warp_inclusive_scan(rej, OpSum());
                    const uint32_t wr = shfl_idx(rincl, 31);
                    uint32_t rr = wk + rincl - rej;
#pragma unroll
                    for (int j = 0; j < ITEMS; ++j) {
                        const int i = r0 + j;
                        if (i < 0 || i >= (int)len) continue;
                        if (f >> j & 1u) wsm[rk++] = x[j];
                        else wsm[rr++] = x[j];
                    }
                    __syncwarp();
                    // the segment's kept total, written by the count pass; the tile's rejected
                    // elements start after the segment's kept run and the earlier tiles'
                    // rejected ones, the warp's after the tile's earlier warps'
                    const uint64_t seg_true = *reinterpret_cast<const uint64_t*>(it.aux);
                    const int first_elem = warp * 32 * ITEMS - (int)mis;  // of the warp's slots
                    const uint32_t before = first_elem <= 0 ? 0u : min((uint32_t)first_elem, len);
                    const uint64_t rej_base = seg_true + (begin - prefix) + (before - wex);
                    for (uint32_t i = lane; i < wk + wr; i += 32) {
                        const uint64_t dst = i < wk ? prefix + wex + i : rej_base + (i - wk);
                        if (dst < it.len) out[dst] = wsm[i];
                        else *err = 3;
                    }
                }
                describe_next();
                __syncthreads();
            }
        }
    }
    if (tid == 0) persistent_exit(b.counters);
}

// ---- host side: buffers, tuner, graphs ------------------------------------------------------------
size_t up256(size_t v) { return (v + 255) / 256 * 256; }

template <typename T>
constexpr int min_tile() {  // the smallest tile of any shape, in elements of T
    return 256 * 3 * (16 / (int)sizeof(T)) - 16 / (int)sizeof(T);
}

// Carves the buffers for S segments and at most `items` work items out of the workspace's
// segment buffer (zeroed when it is (re)allocated).
bool seg_buffers(Workspace& ws, uint64_t S, uint64_t items, SegBuffers* out) {
    const size_t need = 256 + up256((S + 1) * 4) + up256(items * 8) +
                        up256(items * sizeof(ItemDesc));
    char* p = static_cast<char*>(ws.seg(need));
    out->status = static_cast<StatusEntry*>(ws.seg_status(items));
    if (!p || !out->status) return false;
    out->status_cap = ws.seg_status_cap;
    out->counters = reinterpret_cast<uint32_t*>(p);
    p += 256;
    out->item_start = reinterpret_cast<uint32_t*>(p);
    p += up256((S + 1) * 4);
    out->partials = reinterpret_cast<uint64_t*>(p);
    p += up256(items * 8);
    out->items = reinterpret_cast<ItemDesc*>(p);
    return true;
}

struct SegCall {
    int op;            // SegOp
    int red;           // SegRed (reduce)
    DType t;
    SegSrc src;
    uint64_t S;
    uint64_t count;    // CSR: elements of the input array; descriptors: sum of lengths
    uint64_t init_bits;
    bool inclusive;
    bool unique;
    bool tune;         // may time the tile candidates (launches must be idempotent)
    Pred pred;
};

uint64_t items_bound(const SegCall& c, uint64_t tile) { return c.S + c.count / tile + 1; }

template <typename T>
SegPred<T> make_seg_pred(const Pred& p) {
    SegPred<T> e;
    e.kind = p.kind;
    e.negate = p.negate;
    e.c = std::is_floating_point<T>::value ? (T)p.f : std::is_signed<T>::value ? (T)p.i : (T)p.u;
    e.m = (T)p.mod_m;
    e.r = (T)p.mod_r;
    if (std::is_integral<T>::value && sizeof(T) == 4) e.fm = FastMod32::make((int64_t)e.m);
    return e;
}

template <typename T, int BLOCK, int VPT, int OP>
bool launch_kernel(Workspace& ws, const SegArgs<T>& args, const SegBuffers& b, uint64_t items) {
    using Sh = SegShape<T, BLOCK, VPT>;
    auto kfn = k_segmented<T, BLOCK, VPT, OP>;
    const size_t smem = OP == SEG_REDUCE ? 0 : Sh::SMEM;
    if (smem > (48u << 10) && !smem_opt_in<k_segmented<T, BLOCK, VPT, OP>>(smem))
        return cuda_ok(cudaGetLastError(), "segmented shared-memory opt-in");
    // resident CTAs per SM of this instantiation (queried once per device), and no more
    // CTAs than work items: a small batch launches a small grid
    static int per_sm_of[kSmemOptInDevices] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    int& per_sm = per_sm_of[dev < kSmemOptInDevices && dev >= 0 ? dev : 0];
    if (per_sm == 0) {
        int v = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, kfn, BLOCK, smem);
        per_sm = v < 1 ? 1 : v;
    }
    const uint64_t resident = (uint64_t)per_sm * device_info().sm_count;
    const unsigned grid = (unsigned)(items < resident ? items : resident);
    kfn<<<grid ? grid : 1, BLOCK, smem, ws.stream()>>>(args, b, &ws.d_slot->spin_error);
    return cuda_ok(cudaGetLastError(), "segmented launch");
}

template <typename T>
bool launch_fold(Workspace& ws, const SegBuffers& b, uint64_t S, int red) {
    const uint64_t blocks = (S * 32 + 255) / 256;
    k_seg_fold<T><<<(unsigned)(blocks ? blocks : 1), 256, 0, ws.stream()>>>(b, S, red);
    return cuda_ok(cudaGetLastError(), "segmented fold launch");
}

template <typename T, int BLOCK, int VPT>
bool enqueue_shape(Workspace& ws, const SegCall& c, const SegBuffers& b) {
    using Sh = SegShape<T, BLOCK, VPT>;
    constexpr int TILE = Sh::TILE;
    cudaStream_t s = ws.stream();
    volatile int32_t* err = &ws.d_slot->spin_error;
    const uint64_t items_cap = items_bound(c, TILE);
    SegArgs<T> args;
    args.src = c.src;
    args.S = c.S;
    memcpy(&args.init, &c.init_bits, sizeof(T));
    args.inclusive = c.inclusive;
    args.unique = c.unique;
    args.red = c.red;
    args.pred = make_seg_pred<T>(c.pred);
    auto plan = [&](SegEmpty empty) {
        if (items_cap <= kPlanItemsMax) {
            k_seg_plan_items<256><<<1, 256, 0, s>>>(c.src, c.S, c.count, (uint32_t)TILE,
                                                    b.item_start, b.counters, empty,
                                                    nullptr, b.status,
                                                    b.status_cap, err, b.items);
            return;
        }
        k_seg_plan<256><<<1, 256, 0, s>>>(c.src, c.S, c.count, (uint32_t)TILE, b.item_start,
                                          b.counters, empty, nullptr,
                                          b.status, b.status_cap, err, nullptr);
        const uint64_t dg = (items_cap + 255) / 256;
        k_item_descs<<<(unsigned)(dg < 1184 ? dg : 1184), 256, 0, s>>>(c.src, c.S, b.item_start,
                                                                        b.items);
    };
    switch (c.op) {
        case SEG_REDUCE:
            plan(c.red == RED_COUNT ? SegEmpty::ZERO_COUNT : SegEmpty::ZERO_RESULT);
            return launch_kernel<T, BLOCK, VPT, SEG_REDUCE>(ws, args, b, items_cap) &&
                   launch_fold<T>(ws, b, c.S, c.red);
        case SEG_SCAN:
            plan(SegEmpty::NONE);
            return launch_kernel<T, BLOCK, VPT, SEG_SCAN>(ws, args, b, items_cap);
        case SEG_SELECT:
            plan(SegEmpty::ZERO_COUNT);
            return launch_kernel<T, BLOCK, VPT, SEG_SELECT>(ws, args, b, items_cap);
        default: {
            // count pass (per-segment kept totals into the counts), then the scatter; the
            // count pass uses no look-back status, so the scatter takes the plan's epoch
            SegArgs<T> cnt = args;
            cnt.red = RED_COUNT;
            plan(SegEmpty::ZERO_COUNT);
            if (!launch_kernel<T, BLOCK, VPT, SEG_REDUCE>(ws, cnt, b, items_cap) ||
                !launch_fold<T>(ws, b, c.S, RED_COUNT))
                return false;
            return launch_kernel<T, BLOCK, VPT, SEG_PARTITION>(ws, args, b, items_cap);
        }
    }
}

template <typename T>
bool enqueue_typed(Workspace& ws, const SegCall& c, int shape) {
    SegBuffers b;
    if (!seg_buffers(ws, c.S, items_bound(c, min_tile<T>()), &b)) return false;
    switch (shape) {
        case 0: return enqueue_shape<T, 256, 3>(ws, c, b);
        case 1: return enqueue_shape<T, 256, 7>(ws, c, b);
        default: return enqueue_shape<T, 512, 7>(ws, c, b);
    }
}

bool enqueue(Workspace& ws, const SegCall& c, int shape) {
    switch (c.t) {
        case DType::F32: return enqueue_typed<float>(ws, c, shape);
        case DType::F64: return enqueue_typed<double>(ws, c, shape);
        case DType::I32: return enqueue_typed<int32_t>(ws, c, shape);
        case DType::I64: return enqueue_typed<int64_t>(ws, c, shape);
        case DType::U32: return enqueue_typed<uint32_t>(ws, c, shape);
        case DType::U64: return enqueue_typed<uint64_t>(ws, c, shape);
        default: break;
    }
    set_error(PARALLAX_ERR_INVALID_ARGUMENT, "segmented: unsupported element type");
    return false;
}

// ---- autotuner -----------------------------------------------------------------------------------
// Shape per (op, dtype, log2 of the average segment length); timed on the first call with
// those parameters, optionally persisted in PARALLAX_TUNE_CACHE, one line per choice:
// "op dtype bucket block vpt".
std::mutex g_tune_mu;
std::map<std::tuple<int, int, int>, int>* g_tune = nullptr;

int shape_index(int block, int vpt) {
    for (int i = 0; i < kNumShapes; ++i)
        if (kShapes[i].block == block && kShapes[i].vpt == vpt) return i;
    return -1;
}

void tune_load_locked() {
    if (g_tune) return;
    g_tune = new std::map<std::tuple<int, int, int>, int>();
    const char* path = getenv("PARALLAX_TUNE_CACHE");
    if (!path) return;
    FILE* f = fopen(path, "r");
    if (!f) return;
    int op, t, bucket, block, vpt;
    while (fscanf(f, "%d %d %d %d %d", &op, &t, &bucket, &block, &vpt) == 5) {
        const int i = shape_index(block, vpt);
        if (i >= 0) (*g_tune)[std::make_tuple(op, t, bucket)] = i;
    }
    fclose(f);
}

void tune_store_locked() {
    const char* path = getenv("PARALLAX_TUNE_CACHE");
    if (!path) return;
    FILE* f = fopen(path, "w");
    if (!f) return;
    for (auto& kv : *g_tune)
        fprintf(f, "%d %d %d %d %d\n", std::get<0>(kv.first), std::get<1>(kv.first),
                std::get<2>(kv.first), kShapes[kv.second].block, kShapes[kv.second].vpt);
    fclose(f);
}

int bucket_of(const SegCall& c) {
    uint64_t avg = c.S ? c.count / c.S : 0;
    int b = 0;
    while ((1ull << (b + 1)) <= avg && b < 30) ++b;
    return b;
}

// Returns the shape choice, timing the candidates (and leaving valid results) when unknown.
int tuned_shape(Workspace& ws, const SegCall& c) {
    const int opkey = c.op * 8 + c.red * 2 + (c.unique ? 1 : 0);
    const auto key = std::make_tuple(opkey, (int)c.t, bucket_of(c));
    {
        std::lock_guard<std::mutex> g(g_tune_mu);
        tune_load_locked();
        auto it = g_tune->find(key);
        if (it != g_tune->end()) return it->second;
    }
    if (!c.tune || (getenv("PARALLAX_TUNE") && atoi(getenv("PARALLAX_TUNE")) == 0)) {
        const uint64_t avg = c.S ? c.count / c.S : 0;  // untuned: by average segment length
        return avg >= (16u << 10) ? 2 : avg >= (2u << 10) ? 1 : 0;
    }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    int best = 1;
    float best_ms = 1e30f;
    cudaStream_t s = ws.stream();
    for (int cand = 0; cand < kNumShapes; ++cand) {
        if (!enqueue(ws, c, cand)) break;  // warm-up (first-touch, module load)
        cudaEventRecord(e0, s);
        if (!enqueue(ws, c, cand)) break;
        cudaEventRecord(e1, s);
        if (cudaEventSynchronize(e1) != cudaSuccess) break;
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (getenv("PARALLAX_DEBUG"))
            fprintf(stderr, "[parallax] segmented op %d dtype %d bucket %d: %d threads x %d vectors %.3f ms\n",
                    opkey, (int)c.t, bucket_of(c), kShapes[cand].block, kShapes[cand].vpt, ms);
        if (ms < best_ms) {
            best_ms = ms;
            best = cand;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    std::lock_guard<std::mutex> g(g_tune_mu);
    (*g_tune)[key] = best;
    tune_store_locked();
    if (getenv("PARALLAX_DEBUG"))
        fprintf(stderr,
                "[parallax] tuned segmented op %d dtype %d bucket %d -> %d threads x %d vectors "
                "(%.3f ms)\n",
                opkey, (int)c.t, bucket_of(c), kShapes[best].block, kShapes[best].vpt, best_ms);
    return best;
}

// ---- graph capture and replay -----------------------------------------------------------------
std::string graph_key(const SegCall& c, int shape) {
    char k[512];
    snprintf(k, sizeof k, "%d/%d/%d/%d/%llx/%llx/%p/%llx/%llu/%llu/%llx/%d/%d/%d/%g/%lld/%llu/%lld/%lld/%d",
             c.op, c.red, (int)c.unique, (int)c.t, (unsigned long long)c.src.in,
             (unsigned long long)c.src.out, (const void*)c.src.offsets,
             (unsigned long long)c.src.aux, (unsigned long long)c.S, (unsigned long long)c.count,
             (unsigned long long)c.init_bits, (int)c.inclusive, (int)c.pred.kind,
             (int)c.pred.negate, c.pred.f, (long long)c.pred.i, (unsigned long long)c.pred.u,
             (long long)c.pred.mod_m, (long long)c.pred.mod_r, shape);
    return k;
}

const char* op_name(const SegCall& c) {
    switch (c.op) {
        case SEG_REDUCE: return "segmented_reduce";
        case SEG_SCAN: return "segmented_scan";
        case SEG_SELECT: return c.unique ? "segmented_unique" : "segmented_copy_if";
        default: return "segmented_partition";
    }
}

// Sizes the buffers for the smallest tile before any capture (growth would invalidate a
// captured graph).
bool reserve(Workspace& ws, const SegCall& c) {
    SegBuffers b;
    const uint64_t tile = c.t == DType::F64 || c.t == DType::I64 || c.t == DType::U64
        ? (uint64_t)min_tile<uint64_t>() : (uint64_t)min_tile<uint32_t>();
    return seg_buffers(ws, c.S, items_bound(c, tile), &b);
}

bool run(Workspace& ws, const SegCall& c, bool graph) {
    const int shape = tuned_shape(ws, c);
    if (!reserve(ws, c)) return false;
    const size_t es = dtype_size(c.t);
    // algorithmic bytes: input read (+ output written for scans; compaction outputs are
    // data-dependent and partition writes every element)
    const uint64_t bytes = (c.op == SEG_SCAN || c.op == SEG_PARTITION ? 2 : 1) * c.count * es;
    ProfScope prof(ws, op_name(c), bytes);
    {  // planner (+ item descriptors unless it writes them) + the pass(es) (+ the fold)
        const uint64_t V = 16 / es;
        const uint64_t tile = (uint64_t)kShapes[shape].block * kShapes[shape].vpt * V - V;
        const int plan = items_bound(c, tile) <= kPlanItemsMax ? 1 : 2;
        count_launch(plan + (c.op == SEG_PARTITION ? 3 : c.op == SEG_REDUCE ? 2 : 1));
    }
    if (!graph) return enqueue(ws, c, shape);
    return graph_launch(ws, graph_key(c, shape), [&] { return enqueue(ws, c, shape); });
}

int seg_entry(SegCall c, const void* in, void* out, const uint64_t* offsets, void* aux,
              const char* fn) {
    set_ok();
    Workspace* ws = workspace();
    if (!ws) return PARALLAX_ERR_NO_DEVICE;
    if (c.S == 0) return PARALLAX_OK;
    // with count == 0 every segment is empty: the data pointers are never touched and may
    // be null; offsets, results and counts are still read or written
    const bool data = c.count != 0;
    const void* d_in = nullptr;
    void* d_out = nullptr;
    if (data && !(d_in = device_operand(in, fn, "input"))) return last_error();
    const void* d_off = device_operand(offsets, fn, "offsets");
    if (!d_off) return last_error();
    if (c.op != SEG_REDUCE && data && !(d_out = device_operand(out, fn, "output"))) return last_error();
    void* d_aux = nullptr;  // results (reduce) or counts (compaction); scans have none
    if (c.op != SEG_SCAN &&
        !(d_aux = device_operand(aux, fn, c.op == SEG_REDUCE ? "results" : "counts")))
        return last_error();
    if (c.S >= 0xffffffffull || c.count / 1000 + c.S >= 0xffffffffull) {
        set_error(PARALLAX_ERR_INVALID_ARGUMENT, "%s: too many segments / elements", fn);
        return PARALLAX_ERR_INVALID_ARGUMENT;
    }
    const uint32_t es = (uint32_t)dtype_size(c.t);
    const uint32_t aux_stride = c.op == SEG_REDUCE && c.red != RED_COUNT ? es : 8u;
    c.src = SegSrc{static_cast<const uint64_t*>(d_off), nullptr, (uint64_t)d_in, (uint64_t)d_out,
                   (uint64_t)d_aux, aux_stride, es};
    if (!run(*ws, c, true)) return last_error() ? last_error() : PARALLAX_ERR_CUDA;
    return ws->async ? PARALLAX_OK : sync_stream(*ws);
}

Handle* seg_handle(parallax_kernel_t k) { return as_handle(k); }

}  // namespace

bool launch_segmented_descs(Workspace& ws, SegKind op, DType t, const Pred& p, bool inclusive,
                            uint64_t init_bits, const SegDesc* d_descs, uint64_t S,
                            uint64_t total, RedOp red, CompactMode mode) {
    if (S == 0) return true;
    if (S >= 0xffffffffull || total / 1000 + S >= 0xffffffffull) {
        set_error(PARALLAX_ERR_INVALID_ARGUMENT, "batched launch: too many segments / elements");
        return false;
    }
    SegCall c{};
    c.op = op == SegKind::REDUCE ? SEG_REDUCE
         : op == SegKind::SCAN ? SEG_SCAN
         : mode == CompactMode::PARTITION ? SEG_PARTITION : SEG_SELECT;
    c.red = red == RedOp::MAX ? RED_MAX : red == RedOp::MIN ? RED_MIN : RED_SUM;
    c.unique = op == SegKind::COPY_IF && mode == CompactMode::UNIQUE;
    c.t = t;
    c.src = SegSrc{nullptr, d_descs, 0, 0, 0, 0, (uint32_t)dtype_size(t)};
    c.S = S;
    c.count = total;
    c.init_bits = init_bits;
    c.inclusive = inclusive;
    c.tune = false;
    c.pred = p;
    return run(ws, c, false);
}

void* device_operand(const void* p, const char* fn, const char* what) {
    if (!p) {
        set_error(PARALLAX_ERR_INVALID_ARGUMENT, "%s: %s is null", fn, what);
        return nullptr;
    }
    if (arena_contains(p)) {
        ArenaBlock blk;
        if (arena_find(p, &blk) && arena_zero_copy())  // whole-heap capture: in place
            return arena_make_accessible() ? arena_dev(p) : nullptr;
        if (!arena_find(p, &blk) || blk.residency != PARALLAX_DEVICE_RESIDENT) {
            set_error(PARALLAX_ERR_INVALID_ARGUMENT,
                      "%s: %s: arena blocks must be PARALLAX_DEVICE_RESIDENT", fn, what);
            return nullptr;
        }
        return arena_dev(p);
    }
    cudaPointerAttributes attr;
    if (cudaPointerGetAttributes(&attr, p) == cudaSuccess &&
        (attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged))
        return attr.devicePointer ? attr.devicePointer : const_cast<void*>(p);
    cudaGetLastError();
    set_error(PARALLAX_ERR_INVALID_ARGUMENT, "%s: %s must be device memory", fn, what);
    return nullptr;
}

}  // namespace pxb

using namespace pxb;

PXB_EXPORT int parallax_segmented_reduce(parallax_kernel_t kernel, const void* data, size_t count,
                                         const uint64_t* offsets, size_t num_segments,
                                         void* results) {
    Handle* h = seg_handle(kernel);
    if (!h || h->kind != Kind::REDUCE) {
        set_error(PARALLAX_ERR_INVALID_HANDLE, "parallax_segmented_reduce: needs a reduce handle");
        return PARALLAX_ERR_INVALID_HANDLE;
    }
    SegCall c{};
    c.op = SEG_REDUCE;
    c.red = h->op == RedOp::MAX ? RED_MAX : h->op == RedOp::MIN ? RED_MIN : RED_SUM;
    c.t = h->dtype;
    c.count = count;
    c.S = num_segments;
    c.tune = true;
    return seg_entry(c, data, nullptr, offsets, results, "parallax_segmented_reduce");
}

namespace {
int seg_scan_entry(parallax_kernel_t kernel, const void* input, void* output, size_t count,
                   const uint64_t* offsets, size_t num_segments, const void* init,
                   bool inclusive, const char* fn) {
    Handle* h = seg_handle(kernel);
    if (!h || h->kind != Kind::SCAN) {
        set_error(PARALLAX_ERR_INVALID_HANDLE, "%s: needs a scan handle", fn);
        return PARALLAX_ERR_INVALID_HANDLE;
    }
    SegCall c{};
    c.op = SEG_SCAN;
    c.t = h->dtype;
    c.count = count;
    c.S = num_segments;
    c.inclusive = inclusive;
    c.tune = input != output;  // timing the candidates in place would scan twice
    if (init && !inclusive) memcpy(&c.init_bits, init, dtype_size(h->dtype));
    return seg_entry(c, input, output, offsets, nullptr, fn);
}

int seg_compact_entry(parallax_kernel_t kernel, const void* input, void* output, size_t count,
                      const uint64_t* offsets, size_t num_segments, uint64_t* counts,
                      int which, const char* fn) {
    // which: 0 copy_if / remove_if, 1 partition, 2 unique
    Handle* h = seg_handle(kernel);
    const bool ok = h && ((which == 0 && h->kind == Kind::COMPACT_FLAGS) ||
                          (which == 1 && h->kind == Kind::PARTITION_SCATTER) ||
                          (which == 2 && h->kind == Kind::UNIQUE_FLAGS));
    if (!ok) {
        set_error(PARALLAX_ERR_INVALID_HANDLE, "%s: needs a %s handle", fn,
                  which == 0 ? "copy_if / remove_if" : which == 1 ? "partition" : "unique");
        return PARALLAX_ERR_INVALID_HANDLE;
    }
    SegCall c{};
    c.op = which == 1 ? SEG_PARTITION : SEG_SELECT;
    c.unique = which == 2;
    c.t = h->dtype;
    c.count = count;
    c.S = num_segments;
    c.tune = which != 1 || input != output;
    c.pred = h->pred;
    if (h->kind == Kind::COMPACT_FLAGS && h->remove) c.pred.negate = !c.pred.negate;
    return seg_entry(c, input, output, offsets, counts, fn);
}
}  // namespace

PXB_EXPORT int parallax_segmented_exclusive_scan(parallax_kernel_t kernel, const void* input,
                                                 void* output, size_t count,
                                                 const uint64_t* offsets, size_t num_segments,
                                                 const void* init) {
    return seg_scan_entry(kernel, input, output, count, offsets, num_segments, init, false,
                          "parallax_segmented_exclusive_scan");
}

PXB_EXPORT int parallax_segmented_inclusive_scan(parallax_kernel_t kernel, const void* input,
                                                 void* output, size_t count,
                                                 const uint64_t* offsets, size_t num_segments) {
    return seg_scan_entry(kernel, input, output, count, offsets, num_segments, nullptr, true,
                          "parallax_segmented_inclusive_scan");
}

PXB_EXPORT int parallax_segmented_copy_if(parallax_kernel_t kernel, const void* input,
                                          void* output, size_t count, const uint64_t* offsets,
                                          size_t num_segments, uint64_t* counts) {
    return seg_compact_entry(kernel, input, output, count, offsets, num_segments, counts, 0,
                             "parallax_segmented_copy_if");
}

PXB_EXPORT int parallax_segmented_partition(parallax_kernel_t kernel, const void* input,
                                            void* output, size_t count, const uint64_t* offsets,
                                            size_t num_segments, uint64_t* counts) {
    return seg_compact_entry(kernel, input, output, count, offsets, num_segments, counts, 1,
                             "parallax_segmented_partition");
}

PXB_EXPORT int parallax_segmented_unique(parallax_kernel_t kernel, const void* input,
                                         void* output, size_t count, const uint64_t* offsets,
                                         size_t num_segments, uint64_t* counts) {
    return seg_compact_entry(kernel, input, output, count, offsets, num_segments, counts, 2,
                             "parallax_segmented_unique");
}
