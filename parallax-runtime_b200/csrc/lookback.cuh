// Decoupled look-back: the single-pass inter-tile carry shared by the scan and the
// compaction kernels.
//
// Replaces the reference's multi-pass carry (per-block scan -> recursive scan of block
// sums -> add-offsets pass, src/kernel/kernel_launcher.cpp:1280-1342,
// shaders/scan.comp + scan_add.comp). Each tile publishes its aggregate as soon as it is
// known (state AGG) and its inclusive prefix once its look-back completes (state INC).
// A tile's look-back reads its predecessors' status entries, summing aggregates until it
// meets an inclusive prefix. Tiles are processed in blockIdx order (or claimed in order
// from an atomic counter), so every tile a CTA waits on belongs to a CTA that started
// earlier: the waits always end.
// Each wait is still bounded: after `limit` polls (kSpinLimit unless PARALLAX_WAIT_LIMIT
// sets fewer) the kernel records an error code in host-visible memory and carries on with
// a zero contribution, so a fault can never hang the GPU; the host turns the code into
// PARALLAX_ERR_DEVICE_SPIN.
//
// Status entry: 16 bytes, two 8-byte words {low 32 bits of the value, flag} and {high 32
// bits, flag}, written with one 16-byte store and read with one 16-byte load, so a poll is a
// single round trip to L2 (under a saturated memory system that round trip queues behind
// the SM's bulk loads, and it used to take two: flag, then value). Each 8-byte word is
// written and read whole, so the value half in a word always belongs to that word's flag;
// a read whose two flags differ (a load that met the store half-way, or AGG then INC)
// counts as "not published yet" and polls again.
// Flag: bits [31:2] = launch epoch (30 bits), bits [1:0] = state (0 none, 1 AGG, 2 INC).
// Entries left by earlier launches carry an older epoch and read as "none", so the status
// array is never cleared between launches.
#pragma once

#include <string.h>

#include "common.cuh"
#include "runtime.hpp"

namespace pxb {

constexpr uint32_t kSpinLimit = 1u << 22;

// One status entry per tile; the same 16-byte layout for every accumulator type keeps
// flag words at fixed addresses across launches (see Workspace::scratch).
struct __align__(16) StatusEntry {
    uint32_t lo;
    uint32_t flag_lo;
    uint32_t hi;
    uint32_t flag_hi;
};
static_assert(sizeof(StatusEntry) == 16, "status entry layout");

template <typename A>
struct TileStatus {
    StatusEntry* e;
    uint32_t epoch;
    volatile int32_t* err;
    uint32_t limit = kSpinLimit;  // polls of one predecessor before the wait gives up
};

// Poll limit of the look-back waits launched from now on: kSpinLimit, or the smaller
// number of polls given by PARALLAX_WAIT_LIMIT (read once; an opt-in for tests that make
// a wait run out quickly).
uint32_t wait_limit();

template <typename A>
__device__ __forceinline__ void put_val(uint64_t* p, A v) {
    uint64_t bits = 0;
    memcpy(&bits, &v, sizeof(A));
    *p = bits;
}
template <typename A>
__device__ __forceinline__ A get_val(const uint64_t* p) {
    uint64_t bits = (uint64_t)__ldcg(reinterpret_cast<const unsigned long long*>(p));
    A v;
    memcpy(&v, &bits, sizeof(A));
    return v;
}

// Publishes `v` with state 1 (AGG) or 2 (INC) in one 16-byte store.
template <typename A>
__device__ __forceinline__ void publish(StatusEntry* e, uint32_t ep, uint32_t state, A v) {
    uint64_t bits = 0;
    memcpy(&bits, &v, sizeof(A));
    const uint64_t f = (uint64_t)(ep | state) << 32;
    const uint64_t w0 = (bits & 0xffffffffull) | f, w1 = (bits >> 32) | f;
    asm volatile("st.relaxed.gpu.global.v2.u64 [%0], {%1, %2};" ::"l"(e), "l"(w0), "l"(w1)
                 : "memory");
}
// One 16-byte read of an entry: true with its state and value when both flags agree and
// carry this launch's epoch with a published state.
template <typename A>
__device__ __forceinline__ bool read_status(const StatusEntry* e, uint32_t ep, uint32_t* state,
                                            A* v) {
    uint64_t w0, w1;
    asm volatile("ld.relaxed.gpu.global.v2.u64 {%0, %1}, [%2];" : "=l"(w0), "=l"(w1) : "l"(e)
                 : "memory");
    const uint32_t f0 = (uint32_t)(w0 >> 32), f1 = (uint32_t)(w1 >> 32);
    if (f0 != f1 || (f0 & ~3u) != ep || (f0 & 3u) == 0u) return false;
    const uint64_t bits = (w0 & 0xffffffffull) | (w1 << 32);
    memcpy(v, &bits, sizeof(A));
    *state = f0 & 3u;
    return true;
}

// Waits (bounded) until predecessor idx has published, then returns its state (1 AGG,
// 2 INC) and value; a wait that gives up records the error and reads as INC with value 0.
template <typename A>
__device__ __forceinline__ uint32_t poll_status(const TileStatus<A>& ts, int64_t idx, uint32_t ep,
                                                A* v) {
    uint32_t state = 0, spins = 0;
    while (!read_status(&ts.e[idx], ep, &state, v)) {
        if (++spins > ts.limit) {
            *ts.err = 1;
            *v = A(0);
            return 2u;
        }
        if (spins > 8) nanosleep_ns(64);
    }
    return state;
}

// CTA-wide look-back: called by ALL threads of a CTA of BLOCK threads (a multiple of 32),
// with the tile aggregate in every thread. Each round, every thread inspects one
// predecessor (tile - 1 - tid - round offset), so one round trip to L2 covers BLOCK
// predecessors instead of 32: when hundreds of resident tiles stand between a tile and the
// nearest published inclusive prefix, this takes one round trip instead of ten.
// `red` is shared scratch of at least BLOCK / 32 + 1 elements of A and `first` of BLOCK / 32
// ints. Returns the exclusive prefix in every thread; the same contribution order for the
// same status pattern, so integer results are exact and fp results deterministic given the
// pattern.
// `lo` is the first index of the chain (0 for a whole array, a segment's first tile for the
// segmented kernels): that tile publishes its inclusive prefix at once, and indices below
// it are never polled.
// NEAR_FIRST: warp 0 alone inspects the 32 nearest predecessors first, and the CTA-wide
// rounds run only when none of them holds an inclusive prefix (measured on B200 with the
// 16-byte entries: 2^28-element scans 0-5 % faster than CTA-wide rounds from the start).
template <typename A, int BLOCK, bool NEAR_FIRST = false>
__device__ __forceinline__ A lookback_cta(const TileStatus<A>& ts, uint64_t tile, A agg, A* red,
                                          int* first, uint64_t lo = 0) {
    constexpr int WARPS = BLOCK / 32;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t ep = (ts.epoch & 0x3fffffffu) << 2;
    if (tile == lo) {
        if (tid == 0) publish(&ts.e[tile], ep, 2u, agg);
        return A(0);
    }
    if (tid == 0) publish(&ts.e[tile], ep, 1u, agg);
    A excl = A(0);
    int64_t pred = (int64_t)tile - 1;
    if constexpr (NEAR_FIRST) {
        if (warp == 0) {
            const int64_t idx = pred - lane;
            A v = A(0);
            const uint32_t state = idx >= (int64_t)lo ? poll_status(ts, idx, ep, &v) : 2u;
            const unsigned m = __ballot_sync(0xffffffffu, state == 2u);
            const int f = m ? __ffs(m) - 1 : 32;
            A c = lane <= f ? v : A(0);
            c = warp_reduce(c, OpSum());
            if (lane == 0) {
                red[0] = c;
                first[0] = m != 0u;
            }
        }
        __syncthreads();
        excl = red[0];
        const bool done = first[0] != 0;
        __syncthreads();  // red / first reusable
        if (done) {
            if (tid == 0) publish(&ts.e[tile], ep, 2u, excl + agg);
            return excl;
        }
        pred -= 32;
    }
    for (;;) {
        const int64_t idx = pred - tid;
        A v = A(0);
        const uint32_t state = idx >= (int64_t)lo ? poll_status(ts, idx, ep, &v) : 2u;
        // nearest inclusive prefix = the lowest thread index holding one
        const unsigned m = __ballot_sync(0xffffffffu, state == 2u);
        if (lane == 0) first[warp] = m ? warp * 32 + __ffs(m) - 1 : BLOCK;
        __syncthreads();
        int nearest = BLOCK;
#pragma unroll
        for (int w = 0; w < WARPS; ++w) nearest = min(nearest, first[w]);
        A c = tid <= nearest ? v : A(0);
        c = warp_reduce(c, OpSum());
        if (lane == 0) red[warp] = c;
        __syncthreads();
        A round = A(0);
#pragma unroll
        for (int w = 0; w < WARPS; ++w) round = round + red[w];
        excl = round + excl;
        __syncthreads();  // red / first reusable
        if (nearest < BLOCK) break;
        pred -= BLOCK;
    }
    if (tid == 0) publish(&ts.e[tile], ep, 2u, excl + agg);
    return excl;
}

// Status entries live after the small scratch region.
template <typename A>
inline TileStatus<A> tile_status_at(char* scratch, uint32_t epoch, int32_t* err) {
    TileStatus<A> ts;
    ts.e = reinterpret_cast<StatusEntry*>(scratch + kScratchSmall);
    ts.epoch = epoch;
    ts.err = err;
    ts.limit = wait_limit();
    return ts;
}

}  // namespace pxb
