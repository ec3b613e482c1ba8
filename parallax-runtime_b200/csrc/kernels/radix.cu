// Ascending sort of large arrays: one-sweep LSD radix sort with 8-bit digits.
//
// Reference: a global bitonic network, one dispatch + fence wait per (k, j) stage
// (src/kernel/kernel_launcher.cpp:1568-1606, shaders/bitonic.comp:15-29).
//
// Keys are ordered as unsigned integers after the order-preserving transform of
// sortkey.cuh, exactly as the merge sort in sort.cu orders them. A sort under a total order
// of the key bits has one result, so both paths return the same bytes.
//
// Method: D. Adinets and D. Merrill, "Onesweep: A Faster Least Significant Digit Radix Sort
// for GPUs" (2022). One upfront kernel counts the histogram of every digit position in a
// single read of the keys. Then each digit pass, lowest digit first, reads and writes the
// keys once:
//   1. a CTA claims the next tile (atomic counter, so every tile it waits on belongs to a
//      CTA that is already running or done) and loads its keys, warp-striped;
//   2. ranks them stably by the current digit, warp by warp: each warp walks its keys in
//      index order and, per 32 keys, groups lanes with equal digits (shared lane masks), so
//      a key's rank is the warp's running count of its digit plus its lower peers;
//   3. publishes the tile's 256 digit counts at once (state AGG), then finds each digit's
//      global offset by decoupled look-back over the per-(tile, digit) words of earlier
//      tiles (one thread per digit) and publishes the inclusive count (state INC); tile 0
//      starts every chain from the exclusive scan of the upfront histogram;
//   4. places the keys in digit order in shared memory and writes each digit's run to
//      its global offset, so a warp's stores cover consecutive addresses.
// Look-back words are 64-bit: [63:42] pass epoch, [41:40] state, [39:0] count. Words of
// earlier passes carry older epochs and read as "not ready", so nothing is cleared between
// passes. Waits are bounded like the other look-backs (lookback.cuh: kSpinLimit).
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../runtime.hpp"
#include "../segplan.cuh"
#include "../sortkey.cuh"
#include "../tiles.cuh"

namespace pxb {
namespace {

constexpr int kBins = 256;
constexpr int kValBits = 40;
constexpr uint64_t kValMask = (uint64_t(1) << kValBits) - 1;
constexpr uint64_t kStAgg = uint64_t(1) << kValBits;
constexpr uint64_t kStInc = uint64_t(2) << kValBits;
constexpr int kEpochShift = 42;
constexpr int kLookWindow = 4;  // predecessor words a look-back step loads at once

template <typename K> struct RadixShape;
// Keys per thread and CTAs per SM of each key size; build-time knobs (-D) for sweeps.
// Measured on 2^26 uint32 keys (digit pass): 16 keys at 3 CTAs/SM 0.327 ms, 16 at 2 0.350,
// 20 at 2 0.329, 24 at 2 0.315 ms (fewer, larger tiles: fewer look-backs; 64 registers,
// no spills).
#ifndef PXB_RADIX_ITEMS32
#define PXB_RADIX_ITEMS32 24
#endif
#ifndef PXB_RADIX_CTAS32
#define PXB_RADIX_CTAS32 2
#endif
// 8-byte keys, 2^26 int64 sort (eight passes) / 122 M-record segmented key-value sort (four):
// 8 keys at 3 CTAs/SM 3.77 / 4.12 ms, 12 at 2 3.50 / 3.99, 16 at 2 3.42 / 4.05 ms (64
// registers, no spills; 16 x 8 B is the largest tile two CTAs per SM can stage).
#ifndef PXB_RADIX_ITEMS64
#define PXB_RADIX_ITEMS64 16
#endif
#ifndef PXB_RADIX_CTAS64
#define PXB_RADIX_CTAS64 2
#endif
template <> struct RadixShape<uint32_t> {
    static constexpr int BLOCK = 512, ITEMS = PXB_RADIX_ITEMS32, CTAS = PXB_RADIX_CTAS32;
};
template <> struct RadixShape<uint64_t> {
    static constexpr int BLOCK = 512, ITEMS = PXB_RADIX_ITEMS64, CTAS = PXB_RADIX_CTAS64;
};

// Each warp may rank its keys as kSubs independent streams (consecutive parts of its keys),
// each with its own count and mask tables, so the dependency chains overlap. Measured on a
// 2^26-key pass: one stream at three CTAs per SM (0.338 ms, some registers spilled to fit)
// beats two streams at two CTAs per SM (0.362 ms) and at three (0.378 ms).
constexpr int kSubs = 1;

template <typename K>
constexpr size_t radix_smem() {
    return (size_t)RadixShape<K>::BLOCK * RadixShape<K>::ITEMS * sizeof(K) +
           (size_t)(RadixShape<K>::BLOCK / 32) * kSubs * kBins * sizeof(uint32_t) +
           (size_t)RadixShape<K>::BLOCK * RadixShape<K>::ITEMS * sizeof(uint16_t);
}

template <typename K>
__device__ __forceinline__ uint32_t digit_of(K k, int shift) {
    return (uint32_t)(k >> shift) & 0xffu;
}

__device__ __forceinline__ uint64_t ld_relaxed_u64(const uint64_t* p) {
    uint64_t v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed_u64(uint64_t* p, uint64_t v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
// Which 32-bit half of a ranking-table word holds the lane mask of digit d (1 = high).
__device__ __forceinline__ uint32_t mask_half(uint32_t d) { return (d >> 4) & 1u; }

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// ---- upfront histogram ----------------------------------------------------------------------
// Counts, for every digit position p, how many keys have each digit value, in one read of
// the keys. Shared-memory atomics are the limit here, and what they cost is bank conflicts:
// each lane counts into its own copy of the histograms, laid out [p][digit][copy] with
// copy = lane % COPIES, so with 32 copies lane l always hits bank l (conflict-free) and
// with 16 copies at most two lanes share a bank. The host sizes the grid so that every
// per-CTA count stays below 2^32.
template <typename K> struct HistShape;
template <> struct HistShape<uint32_t> { static constexpr int COPIES = 32, U = 16; };
template <> struct HistShape<uint64_t> { static constexpr int COPIES = 16, U = 8; };
constexpr int kHistBlock = 1024;

template <typename K>
constexpr size_t hist_smem() {
    return (size_t)sizeof(K) * kBins * HistShape<K>::COPIES * sizeof(uint32_t);
}

template <typename K, int XF>
__global__ void __launch_bounds__(kHistBlock)
    k_radix_hist(const K* __restrict__ in, uint64_t n, unsigned long long* __restrict__ hist) {
    constexpr int P = sizeof(K);
    constexpr int COPIES = HistShape<K>::COPIES, U = HistShape<K>::U;
    extern __shared__ __align__(16) uint32_t sh[];  // [P][kBins][COPIES]
    for (int i = threadIdx.x; i < P * kBins * COPIES; i += kHistBlock) sh[i] = 0u;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    uint32_t* const mine = sh + (lane % COPIES);
    const uint64_t stride = (uint64_t)gridDim.x * kHistBlock;
    uint64_t i = (uint64_t)blockIdx.x * kHistBlock + threadIdx.x;
    for (; i + (U - 1) * stride < n; i += U * stride) {
        K k[U];
#pragma unroll
        for (int u = 0; u < U; ++u) k[u] = to_key<K, XF>(__ldcs(in + i + u * stride));
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
            for (int p = 0; p < P; ++p)
                atomicAdd(mine + (p * kBins + digit_of(k[u], 8 * p)) * COPIES, 1u);
    }
    for (; i < n; i += stride) {
        const K k = to_key<K, XF>(in[i]);
#pragma unroll
        for (int p = 0; p < P; ++p) atomicAdd(mine + (p * kBins + digit_of(k, 8 * p)) * COPIES, 1u);
    }
    __syncthreads();
    // one (position, digit) row per thread; copies read in a lane-rotated order so a warp's
    // 32 rows hit 32 different banks
    for (int j = threadIdx.x; j < P * kBins; j += kHistBlock) {
        uint32_t v = 0;
#pragma unroll 8
        for (int c = 0; c < COPIES; ++c) v += sh[j * COPIES + ((c + lane) % COPIES)];
        if (v) atomicAdd(&hist[j], (unsigned long long)v);
    }
}

// Exclusive scan over the 256 digits held by threads 0..255 (one value each); every thread
// of the CTA calls it (threads 256.. pass zero). `part` is shared scratch of 8 elements.
template <typename T, int BLOCK>
__device__ __forceinline__ T digit_exclusive_scan(T v, T* part) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const T inc = warp_inclusive_scan(v, OpSum());
    if (warp < kBins / 32 && lane == 31) part[warp] = inc;
    __syncthreads();
    T before = T(0);
    if (warp < kBins / 32)
        for (int w = 0; w < warp; ++w) before += part[w];
    __syncthreads();  // part may be reused by the caller's next scan
    return before + inc - v;
}

// Segmented mode of a digit pass (many segments, each sorted on its own, in one launch): the
// claimed tile is work item `tile` of the planner's list (segplan.cuh), i.e. tile k of one
// segment; offsets are segment-local, the look-back stops at the segment's first tile, and
// that tile starts every digit's chain from the segment's own histogram.
struct SegRadix {
    SegSrc src;                   // segments: data at in_addr, temporary at aux_addr
    const uint32_t* item_start;   // S + 1: first work item of every segment
    const uint32_t* item_seg;     // work item -> segment
    const uint32_t* seg_hist;     // [S][npos][256] digit counts of every segment
    const uint32_t* epoch_base;   // this call's first pass epoch (device side)
    uint64_t S;
    uint32_t npos, pos;           // digit positions counted, this pass's position among them
    uint32_t parity;              // 0: data -> temporary, 1: temporary -> data
};

// ---- one digit pass --------------------------------------------------------------------------
// XF_IN transforms keys as they are read (the first pass reads the caller's values),
// XF_OUT restores them as they are written (the last pass writes the caller's values).
template <typename K, int XF_IN, int XF_OUT, bool SEG = false>
__global__ void __launch_bounds__(RadixShape<K>::BLOCK, RadixShape<K>::CTAS)
    k_radix_pass(const K* __restrict__ in_, K* __restrict__ out_, uint64_t n_, int shift,
                 const unsigned long long* __restrict__ hist, uint64_t* status, uint32_t epoch_,
                 uint64_t tiles, uint32_t* counters, volatile int32_t* err, SegRadix sr) {
    constexpr int BLOCK = RadixShape<K>::BLOCK, ITEMS = RadixShape<K>::ITEMS;
    constexpr int TILE = BLOCK * ITEMS, WARPS = BLOCK / 32;
    constexpr int TABLES = WARPS * kSubs, STREAM_ITEMS = ITEMS / kSubs;
    static_assert(BLOCK >= kBins, "one thread per digit");
    static_assert(ITEMS % kSubs == 0, "whole streams");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    K* const s_keys = reinterpret_cast<K*>(smem_raw);
    uint32_t* const s_wh = reinterpret_cast<uint32_t*>(smem_raw + (size_t)TILE * sizeof(K));
    // each key's rank within its stream, at the key's tile position (kept out of registers)
    uint16_t* const s_rank = reinterpret_cast<uint16_t*>(s_wh + TABLES * kBins);
    __shared__ uint64_t s_goff[kBins];
    __shared__ uint32_t s_goff32[kBins];
    __shared__ uint64_t s_part64[kBins / 32];
    __shared__ uint32_t s_part32[kBins / 32];
    __shared__ uint32_t s_tile;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) s_tile = atomicAdd(&counters[0], 1u);
    // offsets of stream s of this warp in the tile, per digit (filled in step 3a): wh + s * kBins
    uint32_t* const wh = s_wh + warp * kSubs * kBins;
    // the ranking's tables borrow the key buffer, which is free until step 4a: one 64-bit
    // word per (stream, digit) holding the stream's running count of the digit and the lane
    // mask of the current item's peers, so one load reads both. The mask is the low half for
    // digits with bit 4 clear and the high half otherwise: digit d's word spans banks 2d and
    // 2d + 1 (mod 32), so the atomic ORs of a warp spread over all 32 banks, not 16.
    static_assert((size_t)TILE * sizeof(K) >= (size_t)TABLES * kBins * 8, "rank tables fit");
    uint64_t* const wm = reinterpret_cast<uint64_t*>(s_keys) + warp * kSubs * kBins;
#pragma unroll
    for (int i = lane; i < kSubs * kBins; i += 32) wm[i] = 0ull;
    __syncthreads();
    const uint64_t tile = s_tile;
    // plain: tile `tile` of the array; segmented: work item `tile` is tile tk of segment seg
    const K* in = in_;
    K* out = out_;
    uint64_t n = n_, tk = tile, seg = 0;  // tk: tile index within the array / segment
    uint32_t epoch = epoch_;
    if constexpr (SEG) {
        if (tile >= sr.item_start[sr.S]) {  // the grid is an upper bound of the work items
            if (tid == 0) persistent_exit(counters);
            return;
        }
        seg = sr.item_seg[tile];
        tk = tile - sr.item_start[seg];
        n = sr.src.len(seg);
        if (n < 2) {  // sorted already; such a segment may come without a temporary
            if (tid == 0) persistent_exit(counters);
            return;
        }
        const uint64_t a = sr.src.in_addr(seg), b = sr.src.aux_addr(seg);
        in = reinterpret_cast<const K*>(sr.parity ? b : a);
        out = reinterpret_cast<K*>(sr.parity ? a : b);
        epoch = *sr.epoch_base + sr.pos;
    } else if (tile >= tiles) {  // claim counter out of step: touch nothing
        if (tid == 0) {
            *err = kErrRadixRange;
            persistent_exit(counters);
        }
        return;
    }
    const uint64_t base = tk * TILE;
    const uint64_t rem = n - base;
    const uint32_t valid = rem < (uint64_t)TILE ? (uint32_t)rem : (uint32_t)TILE;

    // 1. keys of warp w: tile positions [w * 32 * ITEMS, (w + 1) * 32 * ITEMS), item i of
    // lane l at w * 32 * ITEMS + 32 i + l, so items walked in order visit keys in index order
    K k[ITEMS];
    const uint32_t w0 = (uint32_t)warp * 32 * ITEMS + lane;
    if (valid == (uint32_t)TILE) {
#pragma unroll
        for (int i = 0; i < ITEMS; ++i) k[i] = to_key<K, XF_IN>(__ldcs(in + base + w0 + 32 * i));
    } else {
#pragma unroll
        for (int i = 0; i < ITEMS; ++i) {
            const uint32_t li = w0 + 32 * i;  // padding: the largest key, digit 255 at the end
            k[i] = li < valid ? to_key<K, XF_IN>(in[base + li]) : ~K(0);
        }
    }

    // 2. stable warp-level ranking by the current digit. Lanes holding the same digit find
    // each other through a per-stream table of 256 lane masks (shared-memory atomic OR of
    // the lane's bit into the low half of the digit's word, read back together with the
    // count in the high half, then the group's highest lane writes count + peers with a
    // cleared mask); a key's rank is the stream's running count of its digit plus its lower
    // peers. This keeps the ranking off the SM's narrow branch unit (where match-any issues)
    // and off the ALU (eight ballots per key cost more than the whole pass), with three
    // shared-memory accesses per key.
    static_assert(32 * STREAM_ITEMS <= 0xffff, "ranks fit 16 bits");

    const uint32_t lt = lanemask_lt();
    const uint32_t le = lt | (1u << lane);
#pragma unroll
    for (int j = 0; j < STREAM_ITEMS; ++j) {  // item j of every stream
        uint32_t d[kSubs], peers[kSubs], c[kSubs], ms[kSubs];
#pragma unroll
        for (int t = 0; t < kSubs; ++t) {
            const uint32_t dg = digit_of(k[t * STREAM_ITEMS + j], shift);
            d[t] = dg + t * kBins;
            ms[t] = mask_half(dg);
            atomicOr(reinterpret_cast<uint32_t*>(&wm[d[t]]) + ms[t], 1u << lane);
        }
        __syncwarp();
#pragma unroll
        for (int t = 0; t < kSubs; ++t) {
            const uint64_t v = wm[d[t]];
            peers[t] = (uint32_t)(v >> (32 * ms[t]));
            c[t] = (uint32_t)(v >> (32 - 32 * ms[t])) + __popc(peers[t] & lt);
        }
        __syncwarp();
#pragma unroll
        for (int t = 0; t < kSubs; ++t)  // the highest peer: count + peers, mask cleared
            if ((peers[t] & ~le) == 0) wm[d[t]] = (uint64_t)(c[t] + 1) << (32 - 32 * ms[t]);
        __syncwarp();
#pragma unroll
        for (int t = 0; t < kSubs; ++t) {
            const int i = t * STREAM_ITEMS + j;
            s_rank[w0 + 32 * i] = (uint16_t)c[t];
        }
    }
    __syncthreads();

    // 3a. per digit: counts of the streams -> exclusive over streams (in key order); tile
    // count; publish AGG. Then the digit's start in the tile is added to every stream's
    // offset, so step 4a finds a key's slot with one table read.
    uint32_t cnt = 0;
    if (tid < kBins) {
        const uint64_t* const all = reinterpret_cast<const uint64_t*>(s_keys);
#pragma unroll 8
        for (int w = 0; w < TABLES; ++w) {
            const uint32_t c = (uint32_t)(all[w * kBins + tid] >> (32 - 32 * mask_half(tid)));
            s_wh[w * kBins + tid] = cnt;
            cnt += c;
        }
        if (tk != 0)
            st_relaxed_u64(&status[tile * kBins + tid],
                           ((uint64_t)epoch << kEpochShift) | kStAgg | cnt);
    }
    const uint32_t loc = digit_exclusive_scan<uint32_t, BLOCK>(tid < kBins ? cnt : 0u, s_part32);
    uint64_t start = 0;  // first tile: the digit's first output position
    if (tk == 0) {
        uint64_t h = 0;
        if (tid < kBins) {
            if constexpr (SEG) h = sr.seg_hist[(seg * sr.npos + sr.pos) * kBins + tid];
            else h = hist[tid];
        }
        start = digit_exclusive_scan<uint64_t, BLOCK>(h, s_part64);
    }
    if (tid < kBins) {
#pragma unroll 8
        for (int w = 0; w < TABLES; ++w) s_wh[w * kBins + tid] += loc;
    }
    __syncthreads();

    // 4a. keys in digit order in shared memory
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) {
        const uint32_t r = s_rank[w0 + 32 * i];
        const uint32_t d = digit_of(k[i], shift);
        s_keys[wh[(i / STREAM_ITEMS) * kBins + d] + r] = k[i];
    }

    // 3b. look-back, one thread per digit. The words of the kLookWindow nearest unvisited
    // predecessors are loaded together, so one round trip to L2 covers several tiles; they
    // are then consumed in order until an inclusive count ends the walk.
    if (tid < kBins) {
        uint64_t excl = start;
        if (tk != 0) {  // (segmented: the walk ends at the segment's first tile, always INC)
            bool done = false;
            for (int64_t j = (int64_t)tile - 1; !done && j >= 0; j -= kLookWindow) {
                uint64_t w[kLookWindow];
#pragma unroll
                for (int q = 0; q < kLookWindow; ++q)
                    w[q] = j - q >= 0 ? ld_relaxed_u64(&status[(uint64_t)(j - q) * kBins + tid]) : 0;
#pragma unroll
                for (int q = 0; q < kLookWindow; ++q) {
                    if (done || j - q < 0) break;
                    uint64_t v = w[q];
                    uint32_t spins = 0;
                    while (!((uint32_t)(v >> kEpochShift) == epoch && (v & (kStAgg | kStInc)))) {
                        if (++spins > kSpinLimit) {
                            *err = 1;
                            done = true;
                            break;
                        }
                        if (spins > 8) nanosleep_ns(32);
                        v = ld_relaxed_u64(&status[(uint64_t)(j - q) * kBins + tid]);
                    }
                    if (done) break;
                    excl += v & kValMask;
                    if (v & kStInc) done = true;
                }
            }
        }
        st_relaxed_u64(&status[tile * kBins + tid],
                       ((uint64_t)epoch << kEpochShift) | kStInc | ((excl + cnt) & kValMask));
        // output position of tile-sorted index x: goff[d] + x (excl >= loc always)
        s_goff[tid] = excl - loc;
        s_goff32[tid] = (uint32_t)(excl - loc);
    }
    __syncthreads();

    // 4b. each digit's run to its global offset (32-bit offsets when they fit: one
    // shared-memory wavefront per 32 keys instead of two)
    const bool off32 = n <= 0xffffffffull;
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
        const uint32_t x = (uint32_t)j * BLOCK + tid;
        if (x < valid) {
            const K key = s_keys[x];
            const uint32_t d = digit_of(key, shift);
            const uint64_t pos = off32 ? (uint64_t)(s_goff32[d] + x) : s_goff[d] + x;
            if (pos < n) out[pos] = from_key<K, XF_OUT>(key);
            else *err = kErrRadixRange;
        }
    }
    if (tid == 0) persistent_exit(counters);
}

template <typename K, int XF_IN, int XF_OUT>
bool launch_pass(const K* in, K* out, uint64_t n, int shift, const unsigned long long* hist,
                 uint64_t* status, uint32_t epoch, uint32_t* counters, volatile int32_t* err,
                 uint64_t tiles, cudaStream_t s) {
    constexpr size_t smem = radix_smem<K>();
    if (!smem_opt_in<k_radix_pass<K, XF_IN, XF_OUT>>(smem))
        return cuda_ok(cudaGetLastError(), "k_radix_pass shared-memory opt-in");
    k_radix_pass<K, XF_IN, XF_OUT><<<(unsigned)tiles, RadixShape<K>::BLOCK, smem, s>>>(
        in, out, n, shift, hist, status, epoch, tiles, counters, err, SegRadix{});
    return true;
}

// ---- segmented radix sort -------------------------------------------------------------------
// Digit counts of every segment for digit positions p0 .. P-1. A CTA takes kSegHistItems
// consecutive work items (tiles; consecutive items are mostly of one segment), loads each
// tile's keys into registers before counting them in shared memory (one memory round trip
// per tile), and adds its counts to the segment's histogram with one global atomic per
// nonzero (position, digit) when the segment changes and at its end: a long segment costs
// one flush per kSegHistItems tiles instead of one per tile. seg_hist must be zero on entry.
constexpr int kSegHistBlock = 512;
constexpr int kSegHistItems = 8;

template <typename K, int XF>
__global__ void __launch_bounds__(kSegHistBlock)
    k_seg_radix_hist(SegRadix sr, int p0, uint32_t* __restrict__ seg_hist) {
    constexpr int P = sizeof(K);
    constexpr int TILE = RadixShape<K>::BLOCK * RadixShape<K>::ITEMS;
    constexpr int PER = (TILE + kSegHistBlock - 1) / kSegHistBlock;
    __shared__ uint32_t h[P][kBins];
    const uint32_t total = sr.item_start[sr.S];
    const uint32_t i0 = blockIdx.x * kSegHistItems;
    if (i0 >= total) return;
    const uint32_t i1 = total - i0 < (uint32_t)kSegHistItems ? total : i0 + kSegHistItems;
    const int tid = threadIdx.x;
    const int npos = P - p0;
    for (int i = tid; i < P * kBins; i += kSegHistBlock) (&h[0][0])[i] = 0u;
    __syncthreads();
    auto flush = [&](uint64_t seg) {  // called by the whole CTA (segment ids are uniform)
        __syncthreads();
        for (int i = tid; i < npos * kBins; i += kSegHistBlock) {
            uint32_t& c = h[p0 + i / kBins][i % kBins];
            if (c) atomicAdd(&seg_hist[(seg * npos + i / kBins) * kBins + i % kBins], c);
            c = 0u;
        }
        __syncthreads();
    };
    uint64_t cur = sr.item_seg[i0];
    for (uint32_t item = i0; item < i1; ++item) {
        const uint64_t seg = sr.item_seg[item];
        if (seg != cur) {
            flush(cur);
            cur = seg;
        }
        const uint64_t len = sr.src.len(seg);
        if (len < 2) continue;  // not sorted (see k_radix_pass)
        const uint64_t k = item - sr.item_start[seg];
        const K* in = reinterpret_cast<const K*>(sr.src.in_addr(seg)) + k * TILE;
        const uint64_t rem = len - k * TILE;
        const uint32_t cnt = rem < (uint64_t)TILE ? (uint32_t)rem : (uint32_t)TILE;
        K key[PER];
#pragma unroll
        for (int j = 0; j < PER; ++j) {
            const uint32_t i = (uint32_t)(tid + j * kSegHistBlock);
            key[j] = i < cnt ? to_key<K, XF>(__ldcs(in + i)) : K(0);
        }
#pragma unroll
        for (int j = 0; j < PER; ++j) {
            if ((uint32_t)(tid + j * kSegHistBlock) >= cnt) break;
            for (int p = p0; p < P; ++p) atomicAdd(&h[p][digit_of(key[j], 8 * p)], 1u);
        }
    }
    flush(cur);
}

// Advances the device-side epoch of the segmented radix words by `npass` (so every replay
// of a captured call uses new epochs) and records this call's first epoch in counters[3].
// When the 22-bit epoch would wrap, the look-back words are cleared first.
__global__ void __launch_bounds__(256)
    k_seg_radix_epoch(uint32_t* counters, uint32_t npass, uint64_t* status, uint64_t words) {
    __shared__ uint32_t s_base;
    __shared__ bool s_wrap;
    if (threadIdx.x == 0) {
        uint32_t e = counters[2];
        if (e == 0) e = 1;  // a zeroed buffer: words of epoch 0 never match
        s_wrap = e + npass >= (1u << (64 - kEpochShift));
        s_base = s_wrap ? 1u : e;
    }
    __syncthreads();
    if (s_wrap)
        for (uint64_t i = threadIdx.x; i < words; i += 256) status[i] = 0ull;
    __syncthreads();
    if (threadIdx.x == 0) {
        counters[2] = s_base + npass;
        counters[3] = s_base;
    }
}

template <typename K, int XF_IN, int XF_OUT>
bool launch_seg_pass(const SegRadix& sr, int shift, uint64_t* status, uint32_t* counters,
                     volatile int32_t* err, uint64_t items_cap, cudaStream_t s) {
    constexpr size_t smem = radix_smem<K>();
    if (!smem_opt_in<k_radix_pass<K, XF_IN, XF_OUT, true>>(smem))
        return cuda_ok(cudaGetLastError(), "k_radix_pass shared-memory opt-in");
    k_radix_pass<K, XF_IN, XF_OUT, true><<<(unsigned)items_cap, RadixShape<K>::BLOCK, smem, s>>>(
        nullptr, nullptr, 0, shift, nullptr, status, 0, items_cap, counters, err, sr);
    return true;
}

// S segments (CSR offsets or descriptors, segplan.cuh), each sorted in place by digit
// positions p0 .. P-1 (p0 = 4 on 8-byte records: stably by the high 32 bits). Launches: the
// planner (+ item map), a histogram clear, the segment histograms, the epoch step and one
// launch per digit pass; all capturable in a CUDA graph (device-side epochs).
template <typename K, int XF>
bool seg_radix_sort_keys(Workspace& ws, SegSrc src, uint64_t count, uint64_t S, int p0,
                         bool graph) {
    constexpr int P = sizeof(K);
    constexpr int TILE = RadixShape<K>::BLOCK * RadixShape<K>::ITEMS;
    const uint64_t items_cap = S + count / TILE + 1;
    const uint32_t npos = (uint32_t)(P - p0);
    if (items_cap >= 0x7fffffffull || (npos % 2) != 0) {
        set_error(PARALLAX_ERR_INVALID_ARGUMENT, "segmented sort: too many tiles");
        return false;
    }
    auto up = [](size_t v) { return (v + 255) / 256 * 256; };
    const bool csr_tmp = src.offsets != nullptr;
    const size_t tmp_bytes = csr_tmp ? up(count * sizeof(K)) : 0;
    const size_t hist_bytes = up(S * npos * kBins * sizeof(uint32_t));
    char* t = static_cast<char*>(ws.temp(tmp_bytes + hist_bytes));
    char* sb = static_cast<char*>(ws.seg(256 + up((S + 1) * 4) + up(items_cap * 4)));
    StatusEntry* st = static_cast<StatusEntry*>(ws.seg_status(1));
    const uint64_t words = items_cap * kBins;
    char* rb = static_cast<char*>(ws.seg_radix(256 + words * 8));
    if (!t || !sb || !st || !rb) return false;
    if (csr_tmp) src.aux = reinterpret_cast<uint64_t>(t);
    src.aux_stride = 0;
    src.elem = sizeof(K);
    uint32_t* plan_counters = reinterpret_cast<uint32_t*>(sb);
    uint32_t* item_start = reinterpret_cast<uint32_t*>(sb + 256);
    uint32_t* item_seg = reinterpret_cast<uint32_t*>(sb + 256 + up((S + 1) * 4));
    uint32_t* seg_hist = reinterpret_cast<uint32_t*>(t + tmp_bytes);
    uint32_t* counters = reinterpret_cast<uint32_t*>(rb);
    uint64_t* status = reinterpret_cast<uint64_t*>(rb + 256);
    volatile int32_t* err = &ws.d_slot->spin_error;
    cudaStream_t s = ws.stream();

    SegRadix sr{};
    sr.src = src;
    sr.item_start = item_start;
    sr.item_seg = item_seg;
    sr.seg_hist = seg_hist;
    sr.epoch_base = counters + 3;
    sr.S = S;
    sr.npos = npos;
    ProfScope prof(ws, "segmented_radix_sort", 2 * count * sizeof(K));
    count_launch(4 + npos);
    auto enqueue = [&]() -> bool {
        k_seg_plan<256><<<1, 256, 0, s>>>(src, S, count, (uint32_t)TILE, item_start, plan_counters,
                                          SegEmpty::NONE, nullptr, st, ws.seg_status_cap, err,
                                          items_cap <= kInlineItems ? item_seg : nullptr);
        if (items_cap > kInlineItems)
            k_seg_map<256><<<seg_map_grid(S), 256, 0, s>>>(item_start, S, item_seg);
        if (!cuda_ok(cudaMemsetAsync(seg_hist, 0, hist_bytes, s), "segment histogram clear"))
            return false;
        k_seg_radix_hist<K, XF>
            <<<(unsigned)((items_cap + kSegHistItems - 1) / kSegHistItems), kSegHistBlock, 0, s>>>(
                sr, p0, seg_hist);
        k_seg_radix_epoch<<<1, 256, 0, s>>>(counters, npos, status, words);
        for (int p = p0; p < P; ++p) {
            SegRadix q = sr;
            q.pos = (uint32_t)(p - p0);
            q.parity = (uint32_t)((p - p0) & 1);
            bool ok;
            if (p == p0 && p == P - 1)
                ok = launch_seg_pass<K, XF, XF>(q, 8 * p, status, counters, err, items_cap, s);
            else if (p == p0)
                ok = launch_seg_pass<K, XF, 0>(q, 8 * p, status, counters, err, items_cap, s);
            else if (p == P - 1)
                ok = launch_seg_pass<K, 0, XF>(q, 8 * p, status, counters, err, items_cap, s);
            else
                ok = launch_seg_pass<K, 0, 0>(q, 8 * p, status, counters, err, items_cap, s);
            if (!ok) return false;
        }
        return cuda_ok(cudaGetLastError(), "segmented radix sort launch");
    };
    if (!graph) return enqueue();
    char key[256];
    snprintf(key, sizeof key, "segradix/%d/%d/%d/%p/%p/%llu/%llu", (int)sizeof(K), XF, p0,
             (const void*)src.in, (const void*)src.offsets, (unsigned long long)S,
             (unsigned long long)count);
    return graph_launch(ws, key, enqueue);
}

// Digit passes p0 .. P-1: p0 = 0 sorts by the whole key; p0 = 4 on 8-byte records sorts
// them stably by their high 32 bits alone (LSD passes are stable), the (key << 32 | value)
// records of a sort_kv handle.
template <typename K, int XF>
bool radix_sort_keys(Workspace& ws, void* d_data, uint64_t n, int p0 = 0) {
    constexpr int P = sizeof(K);
    constexpr int TILE = RadixShape<K>::BLOCK * RadixShape<K>::ITEMS;
    const uint64_t tiles = (n + TILE - 1) / TILE;
    if (tiles > 0x7fffffffull || n > kValMask) {
        set_error(PARALLAX_ERR_INVALID_ARGUMENT, "sort: too many elements");
        return false;
    }
    K* data = static_cast<K*>(d_data);
    K* tmp = static_cast<K*>(ws.temp(n * sizeof(K)));
    if (!tmp) return false;
    // radix buffer: [0, 256) tile claim / exit counters, then P histograms, then the
    // per-(tile, digit) look-back words
    constexpr size_t hist_off = 256, status_off = hist_off + (size_t)P * kBins * 8;
    char* rb = static_cast<char*>(ws.radix(status_off + tiles * kBins * 8));
    if (!rb) return false;
    const uint32_t ep0 = ws.next_radix_epochs(P);
    uint32_t* counters = reinterpret_cast<uint32_t*>(rb);
    auto* hist = reinterpret_cast<unsigned long long*>(rb + hist_off);
    auto* status = reinterpret_cast<uint64_t*>(rb + status_off);
    volatile int32_t* err = &ws.d_slot->spin_error;
    cudaStream_t s = ws.stream();
    if (!cuda_ok(cudaMemsetAsync(hist, 0, (size_t)P * kBins * 8, s), "radix histogram clear"))
        return false;
    {
        // grid: one CTA per SM (the copies fill most of its shared memory), more when needed
        // to keep per-CTA counts below 2^31
        uint64_t grid = (uint64_t)device_info().sm_count;
        const uint64_t need = (n + kHistBlock - 1) / kHistBlock;
        if (grid > need) grid = need;
        const uint64_t min_grid = (n >> 31) + 1;
        if (grid < min_grid) grid = min_grid;
        constexpr size_t hsmem = hist_smem<K>();
        if (!smem_opt_in<k_radix_hist<K, XF>>(hsmem))
            return cuda_ok(cudaGetLastError(), "k_radix_hist shared-memory opt-in");
        ProfScope prof(ws, "k_radix_hist", n * sizeof(K));
        k_radix_hist<K, XF><<<(unsigned)grid, kHistBlock, hsmem, s>>>(data, n, hist);
    }
    count_launch();
    static_assert(P % 2 == 0, "an even number of passes ends in the caller's array");
    for (int p = p0; p < P; ++p) {  // P - p0 is even, so the last pass ends in `data`
        const K* src = ((p - p0) % 2 == 0) ? data : tmp;
        K* dst = ((p - p0) % 2 == 0) ? tmp : data;
        const unsigned long long* hp = hist + (size_t)p * kBins;
        bool ok;
        {
            ProfScope prof(ws, "k_radix_pass", 2 * n * sizeof(K));
            if (p == p0)
                ok = launch_pass<K, XF, 0>(src, dst, n, 8 * p, hp, status, ep0 + p, counters, err,
                                           tiles, s);
            else if (p == P - 1)
                ok = launch_pass<K, 0, XF>(src, dst, n, 8 * p, hp, status, ep0 + p, counters, err,
                                           tiles, s);
            else
                ok = launch_pass<K, 0, 0>(src, dst, n, 8 * p, hp, status, ep0 + p, counters, err,
                                          tiles, s);
        }
        if (!ok) return false;
        count_launch();
    }
    return cuda_ok(cudaGetLastError(), "radix sort launch");
}

}  // namespace

bool launch_segmented_radix_sort(Workspace& ws, DType t, const SegSrc& src, uint64_t count,
                                 uint64_t S, bool by_key, bool graph) {
    if (by_key) {
        if (t != DType::U64) {
            set_error(PARALLAX_ERR_INVALID_ARGUMENT, "segmented sort: by-key sorts 8-byte records");
            return false;
        }
        return seg_radix_sort_keys<uint64_t, 0>(ws, src, count, S, 4, graph);
    }
    switch (t) {
        case DType::U32: return seg_radix_sort_keys<uint32_t, 0>(ws, src, count, S, 0, graph);
        case DType::I32: return seg_radix_sort_keys<uint32_t, 1>(ws, src, count, S, 0, graph);
        case DType::F32: return seg_radix_sort_keys<uint32_t, 2>(ws, src, count, S, 0, graph);
        case DType::U64: return seg_radix_sort_keys<uint64_t, 0>(ws, src, count, S, 0, graph);
        case DType::I64: return seg_radix_sort_keys<uint64_t, 1>(ws, src, count, S, 0, graph);
        case DType::F64: return seg_radix_sort_keys<uint64_t, 2>(ws, src, count, S, 0, graph);
        default: break;
    }
    set_error(PARALLAX_ERR_INVALID_ARGUMENT, "segmented sort: unsupported element type");
    return false;
}

uint64_t segmented_radix_tile(DType t) {
    return dtype_size(t) == 4 ? (uint64_t)RadixShape<uint32_t>::BLOCK * RadixShape<uint32_t>::ITEMS
                              : (uint64_t)RadixShape<uint64_t>::BLOCK * RadixShape<uint64_t>::ITEMS;
}

bool launch_radix_sort(Workspace& ws, DType t, void* d_data, size_t n, bool by_key) {
    if (by_key) {
        if (t != DType::U64) {
            set_error(PARALLAX_ERR_INVALID_ARGUMENT, "sort: by-key sorts 8-byte records");
            return false;
        }
        return radix_sort_keys<uint64_t, 0>(ws, d_data, n, 4);
    }
    switch (t) {
        case DType::U32: return radix_sort_keys<uint32_t, 0>(ws, d_data, n);
        case DType::I32: return radix_sort_keys<uint32_t, 1>(ws, d_data, n);
        case DType::F32: return radix_sort_keys<uint32_t, 2>(ws, d_data, n);
        case DType::U64: return radix_sort_keys<uint64_t, 0>(ws, d_data, n);
        case DType::I64: return radix_sort_keys<uint64_t, 1>(ws, d_data, n);
        case DType::F64: return radix_sort_keys<uint64_t, 2>(ws, d_data, n);
        default: break;
    }
    set_error(PARALLAX_ERR_INVALID_ARGUMENT, "sort: unsupported element type");
    return false;
}

}  // namespace pxb
