// Decoupled look-back: the single-pass inter-tile carry shared by the scan and the
// compaction kernels.
//
// Replaces the reference's multi-pass carry (per-block scan -> recursive scan of block
// sums -> add-offsets pass, src/kernel/kernel_launcher.cpp:1280-1342,
// shaders/scan.comp + scan_add.comp). Each tile publishes its aggregate as soon as it is
// known (state AGG) and its inclusive prefix once its look-back completes (state INC).
// A tile's look-back walks predecessors 32 at a time (one warp), summing aggregates until
// it meets an inclusive prefix. Tiles are processed in blockIdx order, so every tile a
// CTA waits on belongs to a CTA that was dispatched earlier: the waits always end.
// Each wait is still bounded: after kSpinLimit polls the kernel records an error code in
// host-visible memory and carries on with a zero contribution, so a fault can never
// hang the GPU; the host turns the code into PARALLAX_ERR_DEVICE_SPIN.
//
// Status words: bits [31:2] = launch epoch (30 bits), bits [1:0] = state
// (0 none, 1 AGG, 2 INC). Words left by earlier launches carry an older epoch and read as
// "none", so the status array is never cleared between launches.
#pragma once

#include <string.h>

#include "common.cuh"
#include "runtime.hpp"

namespace pxb {

constexpr uint32_t kSpinLimit = 1u << 22;

// One status entry per tile; the same 24-byte layout for every accumulator type keeps
// flag words at fixed addresses across launches (see Workspace::scratch).
struct StatusEntry {
    uint32_t flag;
    uint32_t pad;
    uint64_t agg;
    uint64_t inc;
};
static_assert(sizeof(StatusEntry) == 24, "status entry layout");

template <typename A>
struct TileStatus {
    StatusEntry* e;
    uint32_t epoch;
    volatile int32_t* err;
};

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

// Must be called by all 32 lanes of exactly one warp of the CTA. Returns the exclusive
// prefix (sum of aggregates of tiles 0..tile-1) in every lane.
template <typename A>
__device__ __forceinline__ A lookback(const TileStatus<A>& ts, uint64_t tile, A agg) {
    const int lane = threadIdx.x & 31;
    const uint32_t ep = (ts.epoch & 0x3fffffffu) << 2;
    if (tile == 0) {
        if (lane == 0) {
            put_val(&ts.e[0].inc, agg);
            st_release_u32(&ts.e[0].flag, ep | 2u);
        }
        return A(0);
    }
    if (lane == 0) {
        put_val(&ts.e[tile].agg, agg);
        st_release_u32(&ts.e[tile].flag, ep | 1u);
    }
    A excl = A(0);
    int64_t pred = (int64_t)tile - 1;
    for (;;) {
        const int64_t idx = pred - lane;
        uint32_t state = 2u;
        A v = A(0);
        if (idx >= 0) {
            uint32_t f = 0, spins = 0;
            bool gave_up = false;
            for (;;) {
                f = ld_acquire_u32(&ts.e[idx].flag);
                if ((f & ~3u) == ep && (f & 3u) != 0u) break;
                if (++spins > kSpinLimit) {
                    *ts.err = 1;
                    gave_up = true;
                    break;
                }
                if (spins > 16) nanosleep_ns(64);
            }
            if (gave_up) {
                state = 2u;
            } else {
                state = f & 3u;
                v = state == 2u ? get_val<A>(&ts.e[idx].inc) : get_val<A>(&ts.e[idx].agg);
            }
        }
        const unsigned m = __ballot_sync(0xffffffffu, state == 2u);
        const int first = m ? __ffs(m) - 1 : 32;
        A c = lane <= first ? v : A(0);
        c = warp_reduce(c, OpSum());
        excl = c + excl;
        if (m) break;
        pred -= 32;
    }
    if (lane == 0) {
        put_val(&ts.e[tile].inc, excl + agg);
        st_release_u32(&ts.e[tile].flag, ep | 2u);
    }
    return excl;
}

// CTA-wide look-back: called by ALL threads of a CTA of BLOCK threads (a multiple of 32),
// with the tile aggregate in every thread. Each round, every thread inspects one
// predecessor (tile - 1 - tid - round offset), so one round trip to L2 covers BLOCK
// predecessors instead of 32: when hundreds of resident tiles stand between a tile and the
// nearest published inclusive prefix, this takes a couple of round trips instead of ten.
// `red` is shared scratch of at least BLOCK / 32 + 1 elements of A and `first` of BLOCK / 32
// ints. Returns the exclusive prefix in every thread; the same contribution order for the
// same status pattern, so integer results are exact and fp results deterministic given the
// pattern.
// `lo` is the first index of the chain (0 for a whole array, a segment's first tile for the
// segmented kernels): that tile publishes its inclusive prefix at once, and indices below
// it are never polled.
// Waits (bounded) until predecessor idx has published, then returns its state (1 AGG,
// 2 INC) and value; a wait that gives up records the error and reads as INC with value 0.
template <typename A>
__device__ __forceinline__ uint32_t poll_status(const TileStatus<A>& ts, int64_t idx, uint32_t ep,
                                                A* v) {
    uint32_t f = 0, spins = 0;
    for (;;) {
        f = ld_acquire_u32(&ts.e[idx].flag);
        if ((f & ~3u) == ep && (f & 3u) != 0u) break;
        if (++spins > kSpinLimit) {
            *ts.err = 1;
            *v = A(0);
            return 2u;
        }
        if (spins > 16) nanosleep_ns(64);
    }
    const uint32_t state = f & 3u;
    *v = state == 2u ? get_val<A>(&ts.e[idx].inc) : get_val<A>(&ts.e[idx].agg);
    return state;
}

// NEAR_FIRST: warp 0 alone inspects the 32 nearest predecessors first, and the CTA-wide
// rounds run only when none of them holds an inclusive prefix (in the steady state one of
// them does, and 32 polls cost far less than BLOCK).
template <typename A, int BLOCK, bool NEAR_FIRST = false>
__device__ __forceinline__ A lookback_cta(const TileStatus<A>& ts, uint64_t tile, A agg, A* red,
                                          int* first, uint64_t lo = 0) {
    constexpr int WARPS = BLOCK / 32;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t ep = (ts.epoch & 0x3fffffffu) << 2;
    if (tile == lo) {
        if (tid == 0) {
            put_val(&ts.e[tile].inc, agg);
            st_release_u32(&ts.e[tile].flag, ep | 2u);
        }
        return A(0);
    }
    if (tid == 0) {
        put_val(&ts.e[tile].agg, agg);
        st_release_u32(&ts.e[tile].flag, ep | 1u);
    }
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
            if (tid == 0) {
                put_val(&ts.e[tile].inc, excl + agg);
                st_release_u32(&ts.e[tile].flag, ep | 2u);
            }
            return excl;
        }
        pred -= 32;
    }
    for (;;) {
        const int64_t idx = pred - tid;
        uint32_t state = 2u;
        A v = A(0);
        if (idx >= (int64_t)lo) {
            uint32_t f = 0, spins = 0;
            bool gave_up = false;
            for (;;) {
                f = ld_acquire_u32(&ts.e[idx].flag);
                if ((f & ~3u) == ep && (f & 3u) != 0u) break;
                if (++spins > kSpinLimit) {
                    *ts.err = 1;
                    gave_up = true;
                    break;
                }
                if (spins > 16) nanosleep_ns(64);
            }
            if (!gave_up) {
                state = f & 3u;
                v = state == 2u ? get_val<A>(&ts.e[idx].inc) : get_val<A>(&ts.e[idx].agg);
            }
        }
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
    if (tid == 0) {
        put_val(&ts.e[tile].inc, excl + agg);
        st_release_u32(&ts.e[tile].flag, ep | 2u);
    }
    return excl;
}

// Status entries live after the small scratch region.
template <typename A>
inline TileStatus<A> tile_status_at(char* scratch, uint32_t epoch, int32_t* err) {
    TileStatus<A> ts;
    ts.e = reinterpret_cast<StatusEntry*>(scratch + kScratchSmall);
    ts.epoch = epoch;
    ts.err = err;
    return ts;
}

}  // namespace pxb
