// Single-pass inclusive / exclusive '+' scan.
//
// Reference: block Hillis-Steele scan (8 rounds, 2 barriers each) + recursive scan of the
// block sums + an add-offsets pass, each a separate dispatch with a fence wait
// (src/kernel/kernel_launcher.cpp:1280-1342, shaders/scan.comp:16-35,
// shaders/scan_add.comp:14-19); exclusive adds a shift pass writing
// out[i] = init + incl[i-1] (kernel_launcher.cpp:1346-1475).
//
// Here: one launch, one 512-thread CTA per 112 KiB tile (two per SM), in blockIdx order.
// Each CTA
//   1. stages its tile as two 56 KiB sub-tiles (512 threads x 7 x 16 bytes), one bulk
//      copy (cp.async.bulk) and one mbarrier each, so 112 KiB per CTA are in flight at once
//      and work starts when the first sub-tile lands (tiles.cuh),
//   2. sums 28 (4-byte) or 14 (8-byte) consecutive elements per thread per sub-tile
//      (rows of 112 bytes, an odd number of 16-byte words: conflict-free 128-bit shared
//      loads),
//   3. scans row totals with warp shuffles and the 32 (sub-tile, warp) totals in one warp,
//   4. gets the tile's exclusive prefix by decoupled look-back (lookback.cuh),
//   5. rescans each row, writes results into the staged tile and stores it with one bulk
//      copy.
// HBM traffic is the algorithmic minimum: n*s read + n*s written.
// Accumulation: fp32 data is scanned per thread in fp32 (28 terms per sub-tile) and carried
// across threads, warps and tiles in fp64; integers wrap around in their unsigned type.
#include <stdint.h>
#include <string.h>

#include <mutex>

#include "../lookback.cuh"
#include "../runtime.hpp"
#include "../tiles.cuh"
#include "../tma.cuh"

namespace pxb {
namespace {

// Tile shape, chosen by measurement on B200 (2^28 elements): 112 KiB tiles at two CTAs per
// SM beat 48 KiB tiles at four per SM by 8-10 % (the look-back's fixed latency is paid per
// tile), and 16 KiB or 80 KiB tiles were slower still.
// The shape can be overridden at build time (PXB_SCAN_BLOCK / _VPT / _SUB / _CTAS) to sweep
// it; kSub x (kBlock / 32) must be 32.
#ifndef PXB_SCAN_BLOCK
#define PXB_SCAN_BLOCK 512
#endif
#ifndef PXB_SCAN_VPT
#define PXB_SCAN_VPT 7
#endif
#ifndef PXB_SCAN_SUB
#define PXB_SCAN_SUB 2
#endif
#ifndef PXB_SCAN_CTAS
#define PXB_SCAN_CTAS 2
#endif
constexpr int kBlock = PXB_SCAN_BLOCK;
constexpr int kVpt = PXB_SCAN_VPT;  // 16-byte vectors per thread; odd => conflict-free row reads
constexpr int kCtasPerSm = PXB_SCAN_CTAS;

template <typename T> struct ScanTypes;
template <> struct ScanTypes<float> { using L = float; using A = double; };
template <> struct ScanTypes<double> { using L = double; using A = double; };
template <> struct ScanTypes<int32_t> { using L = uint32_t; using A = uint32_t; };
template <> struct ScanTypes<uint32_t> { using L = uint32_t; using A = uint32_t; };
template <> struct ScanTypes<int64_t> { using L = uint64_t; using A = uint64_t; };
template <> struct ScanTypes<uint64_t> { using L = uint64_t; using A = uint64_t; };

constexpr int kSub = PXB_SCAN_SUB;  // sub-tiles per look-back tile; kSub x warps = 32 lanes

template <typename T>
struct ScanShape {
    static constexpr int V = 16 / sizeof(T);
    static constexpr int ITEMS = kVpt * V;          // elements per thread per sub-tile
    static constexpr int SUB = kBlock * ITEMS;      // 56 KiB sub-tile
    static constexpr int TILE = kSub * SUB;         // 112 KiB look-back tile
    static constexpr size_t SMEM = TILE * sizeof(T);
};

// Phase 1 sums each thread's 112-byte row of every sub-tile as soon as that sub-tile lands;
// one 32-lane scan over the (sub-tile, warp) totals - in element order - gives every
// warp's offset and the tile aggregate; warp 0 runs the look-back. Phase 2 re-reads each
// row from shared memory, scans it and writes the results in place. The caller has
// staged the tile (bulk part arriving on bars[] with `parity`, ragged part filled) and
// stores it afterwards.
template <typename T, bool EXCL, bool BULK>
__device__ __forceinline__ void scan_tile(T* buf, uint64_t* bars, uint32_t parity,
                                          typename ScanTypes<T>::A* s_tot, uint64_t tile,
                                          typename ScanTypes<T>::A init,
                                          const TileStatus<typename ScanTypes<T>::A>& ts,
                                          typename ScanTypes<T>::A* red, int* first,
                                          T* sub_out = nullptr, uint32_t bulk = 0) {
    using L = typename ScanTypes<T>::L;
    using A = typename ScanTypes<T>::A;
    constexpr int V = ScanShape<T>::V;
    constexpr int ITEMS = ScanShape<T>::ITEMS;
    constexpr int SUB = ScanShape<T>::SUB;
    constexpr int WARPS = kBlock / 32;
    static_assert(kSub * WARPS == 32, "one lane per (sub-tile, warp)");
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

    // ---- phase 1: row totals of every sub-tile ----
    A tex[kSub];  // exclusive prefix of this thread's row within its warp, per sub-tile
#pragma unroll
    for (int s = 0; s < kSub; ++s) {
        if constexpr (BULK) wait_bar(&bars[s], parity, ts.err);
        const uint4* row = reinterpret_cast<const uint4*>(buf + s * SUB + tid * ITEMS);
        L sum = L(0);
#pragma unroll
        for (int v = 0; v < kVpt; ++v) {
            const uint4 r = row[v];
            const T* e = reinterpret_cast<const T*>(&r);
#pragma unroll
            for (int k = 0; k < V; ++k) sum = sum + (L)e[k];
        }
        const A incl = warp_inclusive_scan((A)sum, OpSum());
        const A ex = shfl_up(incl, 1);
        tex[s] = lane == 0 ? A(0) : ex;
        if (lane == 31) s_tot[s * WARPS + warp] = incl;
    }
    __syncthreads();
    // Every warp scans the 32 (sub-tile, warp) totals itself (identical shuffle sequence,
    // identical result), then the whole CTA runs the look-back.
    A woff[kSub];  // offset of this warp's rows within the tile, per sub-tile
    A agg;
    {
        const A v = s_tot[lane];
        const A vi = warp_inclusive_scan(v, OpSum());
        agg = shfl_idx(vi, 31);
        A vex = shfl_up(vi, 1);
        if (lane == 0) vex = A(0);
#pragma unroll
        for (int s = 0; s < kSub; ++s) woff[s] = shfl_idx(vex, s * WARPS + warp);
    }
    const A prefix = lookback_cta<A, kBlock, true>(ts, tile, agg, red, first);

    // ---- phase 2: scan each row and write the results in place ----
#pragma unroll
    for (int s = 0; s < kSub; ++s) {
        A tb = (prefix + woff[s]) + tex[s];
        if constexpr (EXCL) tb = init + tb;
        uint4* row = reinterpret_cast<uint4*>(buf + s * SUB + tid * ITEMS);
        L x[ITEMS];
#pragma unroll
        for (int v = 0; v < kVpt; ++v) {
            const uint4 r = row[v];
            const T* e = reinterpret_cast<const T*>(&r);
#pragma unroll
            for (int k = 0; k < V; ++k) x[v * V + k] = (L)e[k];
        }
#pragma unroll
        for (int j = 1; j < ITEMS; ++j) x[j] = x[j - 1] + x[j];
#pragma unroll
        for (int v = 0; v < kVpt; ++v) {
            uint4 r;
            T* e = reinterpret_cast<T*>(&r);
#pragma unroll
            for (int k = 0; k < V; ++k) {
                const int j = v * V + k;
                if constexpr (EXCL) e[k] = (T)(j == 0 ? tb : tb + (A)x[j - 1]);
                else e[k] = (T)(tb + (A)x[j]);
            }
            row[v] = r;
        }
        if constexpr (BULK) {
            // with sub_out: each sub-tile's bulk store leaves as soon as the sub-tile is
            // written, so its shared-memory read overlaps the next sub-tile's rescan
            if (sub_out && s + 1 < kSub) {
                fence_proxy_async_smem();
                __syncthreads();
                const uint32_t lo = (uint32_t)s * SUB, hi = bulk < lo + SUB ? bulk : lo + SUB;
                if (tid == 0 && hi > lo) {
                    bulk_store(sub_out + lo, buf + lo, (hi - lo) * (uint32_t)sizeof(T));
                    bulk_commit();
                }
            }
        }
    }
    if constexpr (BULK) fence_proxy_async_smem();
    __syncthreads();
    if constexpr (BULK) {
        if (sub_out) {
            const uint32_t lo = (uint32_t)(kSub - 1) * SUB;
            if (tid == 0 && bulk > lo) {
                bulk_store(sub_out + lo, buf + lo, (bulk - lo) * (uint32_t)sizeof(T));
                bulk_commit();
            }
        }
    }
}

// One CTA per 112 KiB tile, in blockIdx order: unaligned operands (BULK = false) and the
// allocation-free entry point.
// `tile0` is the first tile of this launch: a scan launched in chunks (so its copies can
// overlap its tiles) passes each chunk's first tile, and every chunk shares one look-back
// epoch, so the first tile of a chunk looks back into the chunks before it.
// With `claim`, a CTA takes its tile from an atomic counter instead of its blockIdx (see
// tile_claim()).
template <typename T, bool EXCL, bool BULK>
__global__ void __launch_bounds__(kBlock, kCtasPerSm)
k_scan(const T* in, T* out, uint64_t n,  // in == out allowed (in-place ABI scan)
       typename ScanTypes<T>::A init, TileStatus<typename ScanTypes<T>::A> ts, uint64_t tile0,
       uint32_t* claim) {
    using A = typename ScanTypes<T>::A;
    constexpr int SUB = ScanShape<T>::SUB;
    constexpr int TILE = ScanShape<T>::TILE;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    T* buf = reinterpret_cast<T*>(smem_raw);
    __shared__ __align__(8) uint64_t bars[kSub];
    __shared__ A s_tot[32];
    __shared__ A s_red[kBlock / 32 + 1];
    __shared__ int s_first[kBlock / 32];
    __shared__ uint32_t s_claim;
    const int tid = threadIdx.x;
    const uint64_t tile = tile0 + (claim ? tile_claim(claim, s_claim) : blockIdx.x);
    const uint64_t base = tile * (uint64_t)TILE;
    const uint64_t rem = n - base;
    const uint32_t cnt = rem < (uint64_t)TILE ? (uint32_t)rem : (uint32_t)TILE;
    const uint32_t bulk = stage_tile<T, SUB, kSub, kBlock, BULK>(buf, bars, in, base, cnt);
    __syncthreads();
    scan_tile<T, EXCL, BULK>(buf, bars, 0, s_tot, tile, init, ts, s_red, s_first,
                             BULK ? out + base : nullptr, bulk);
    for (uint32_t e = bulk + tid; e < cnt; e += kBlock) out[base + e] = buf[e];
    if constexpr (BULK) {
        if (tid == 0 && bulk) bulk_wait_read_all();
    }
    if (claim && tid == 0) persistent_exit(claim);
}

// Persistent CTAs (two per SM) with two tile buffers each: the bulk copies of the next
// claimed tile fill one buffer while the current tile is scanned out of the other, so
// every SM keeps ~96 KiB of loads in flight. Operands 16-byte aligned.
template <typename T, bool EXCL>
__global__ void __launch_bounds__(kBlock, 2)
k_scan_persistent(const T* in, T* out, uint64_t n, uint64_t num_tiles,
                  typename ScanTypes<T>::A init, TileStatus<typename ScanTypes<T>::A> ts,
                  uint32_t* counters) {
    using A = typename ScanTypes<T>::A;
    constexpr int SUB = ScanShape<T>::SUB;
    constexpr int TILE = ScanShape<T>::TILE;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    T* const buf0 = reinterpret_cast<T*>(smem_raw);  // buffer b at buf0 + b * TILE
    __shared__ __align__(8) uint64_t bars[2][kSub];
    __shared__ A s_tot[32];
    __shared__ A s_red[kBlock / 32 + 1];
    __shared__ int s_first[kBlock / 32];
    __shared__ uint32_t s_tile[2];
    const int tid = threadIdx.x;

    if (tid == 0) {
#pragma unroll
        for (int b = 0; b < 2; ++b)
#pragma unroll
            for (int s = 0; s < kSub; ++s) mbar_init(&bars[b][s], 1);
        fence_mbar_init();
        const uint32_t t0 = atomicAdd(&counters[0], 1u);
        s_tile[0] = t0;
        if (t0 < num_tiles) {
            const uint64_t base = (uint64_t)t0 * TILE;
            const uint64_t rem = n - base;
            issue_tile<T, SUB, kSub>(buf0, bars[0], in, base,
                                     rem < (uint64_t)TILE ? (uint32_t)rem : (uint32_t)TILE);
        }
    }
    __syncthreads();
    for (uint32_t it = 0;; ++it) {
        const int b = it & 1;
        const uint32_t parity = (it >> 1) & 1u;
        const uint32_t cur = s_tile[b];
        if (cur >= num_tiles) break;
        if (tid == 0) {  // prefetch: claim the next tile and start its copies
            bulk_wait_read_all();  // the previous tile's store has left the other buffer
            fence_proxy_async_smem();
            const uint32_t nxt = atomicAdd(&counters[0], 1u);
            s_tile[b ^ 1] = nxt;
            if (nxt < num_tiles) {
                const uint64_t nbase = (uint64_t)nxt * TILE;
                const uint64_t nrem = n - nbase;
                issue_tile<T, SUB, kSub>(buf0 + (size_t)(b ^ 1) * TILE, bars[b ^ 1], in, nbase,
                                         nrem < (uint64_t)TILE ? (uint32_t)nrem : (uint32_t)TILE);
            }
        }
        T* buf = buf0 + (size_t)b * TILE;
        const uint64_t base = (uint64_t)cur * TILE;
        const uint64_t rem = n - base;
        const uint32_t cnt = rem < (uint64_t)TILE ? (uint32_t)rem : (uint32_t)TILE;
        const uint32_t bulk = bulk_elems<T>(cnt);
        if (cnt < (uint32_t)TILE || bulk < cnt) {  // the last tile: ragged end and padding
            fill_ragged<T, TILE, kBlock>(buf, in, base, cnt, bulk);
            __syncthreads();
        }
        scan_tile<T, EXCL, true>(buf, bars[b], parity, s_tot, cur, init, ts, s_red, s_first);
        if (tid == 0 && bulk) {
            bulk_store(out + base, buf, bulk * (uint32_t)sizeof(T));
            bulk_commit();
        }
        for (uint32_t e = bulk + tid; e < cnt; e += kBlock) out[base + e] = buf[e];
        __syncthreads();  // s_tile / s_tot / plain reads of buf done before the next round
    }
    if (tid == 0) {
        bulk_wait_read_all();
        persistent_exit(counters);
    }
}

// Launches tiles [tile0, tile0 + count).
template <typename T, bool EXCL, bool BULK>
bool launch_tiles_single(const T* in, T* out, uint64_t n, typename ScanTypes<T>::A init,
                         TileStatus<typename ScanTypes<T>::A> ts, uint64_t count,
                         cudaStream_t s, uint64_t tile0 = 0, uint32_t* claim = nullptr) {
    if (!smem_opt_in<k_scan<T, EXCL, BULK>>(ScanShape<T>::SMEM))
        return cuda_ok(cudaGetLastError(), "k_scan shared-memory opt-in");
    k_scan<T, EXCL, BULK><<<(unsigned)count, kBlock, ScanShape<T>::SMEM, s>>>(
        in, out, n, init, ts, tile0, PXB_TILE_CLAIM ? claim : nullptr);
    return true;
}

template <typename T, bool EXCL>
bool launch_tiles_persistent(const T* in, T* out, uint64_t n, typename ScanTypes<T>::A init,
                             TileStatus<typename ScanTypes<T>::A> ts, uint64_t tiles,
                             uint32_t* counters, cudaStream_t s) {
    constexpr size_t smem = 2 * ScanShape<T>::SMEM;
    if (!smem_opt_in<k_scan_persistent<T, EXCL>>(smem))
        return cuda_ok(cudaGetLastError(), "k_scan_persistent shared-memory opt-in");
    uint64_t grid = 2ull * device_info().sm_count;
    if (grid > tiles) grid = tiles;
    k_scan_persistent<T, EXCL><<<(unsigned)grid, kBlock, smem, s>>>(in, out, n, tiles, init, ts,
                                                                     counters);
    return true;
}

template <typename T>
bool scan_typed(Workspace& ws, bool exclusive, const void* d_in, void* d_out, uint64_t n,
                const void* init_host) {
    using A = typename ScanTypes<T>::A;
    constexpr int TILE = ScanShape<T>::TILE;
    const uint64_t tiles = (n + TILE - 1) / TILE;
    if (tiles > 0x7fffffffull) {
        set_error(PARALLAX_ERR_INVALID_ARGUMENT, "scan: %llu elements exceed the grid limit",
                  (unsigned long long)n);
        return false;
    }
    char* scratch = ws.scratch(tiles);
    if (!scratch) return false;
    auto ts = tile_status_at<A>(scratch, ws.next_epoch(), &ws.d_slot->spin_error);
    A init = A(0);
    if (exclusive && init_host) {
        T v;
        memcpy(&v, init_host, sizeof(T));
        init = (A)v;
    }
    // bulk copies only between HBM and shared memory; operands in the page-locked host
    // mirror (small coherent operands, whole-heap capture) take the plain-load path
    const bool bulk = (reinterpret_cast<uintptr_t>(d_in) % 16 == 0) &&
                      (reinterpret_cast<uintptr_t>(d_out) % 16 == 0) &&
                      !arena_contains(d_in) && !arena_contains(d_out);
    const T* in = static_cast<const T*>(d_in);
    T* out = static_cast<T*>(d_out);
    cudaStream_t s = ws.stream();
    ProfScope prof(ws, exclusive ? "k_scan_exclusive" : "k_scan_inclusive", 2 * n * sizeof(T));
    uint32_t* counters = reinterpret_cast<uint32_t*>(scratch + ScratchOff::counters);
    static const bool persistent = getenv("PARALLAX_PERSISTENT_TILES") != nullptr;
    bool ok;
    if (exclusive) {
        ok = !bulk ? launch_tiles_single<T, true, false>(in, out, n, init, ts, tiles, s, 0, counters)
           : persistent ? launch_tiles_persistent<T, true>(in, out, n, init, ts, tiles, counters, s)
                        : launch_tiles_single<T, true, true>(in, out, n, init, ts, tiles, s, 0, counters);
    } else {
        ok = !bulk ? launch_tiles_single<T, false, false>(in, out, n, init, ts, tiles, s, 0, counters)
           : persistent ? launch_tiles_persistent<T, false>(in, out, n, init, ts, tiles, counters, s)
                        : launch_tiles_single<T, false, true>(in, out, n, init, ts, tiles, s, 0, counters);
    }
    if (!ok) return false;
    count_launch();
    return cuda_ok(cudaGetLastError(), "k_scan launch");
}

// Scan of host arena operands with the copies interleaved with the tiles. The tiles are
// launched in chunks of kCopyChunkTiles on the workspace stream; chunk c's upload runs on
// the workspace's upload stream and chunk c's download on its download stream, ordered by
// events, so while the tiles of chunk c run, chunk c+1 is on its way up and chunk c-1 on its
// way down (the two copy directions run on separate copy engines). All chunks share one
// look-back epoch: the result is the same scan as one launch over every tile.
constexpr uint64_t kCopyChunkTiles = 296;  // two waves of two CTAs per SM: ~33 MB of fp32

template <typename T>
bool scan_copies_typed(Workspace& ws, bool exclusive, const void* h_in, const void* d_in,
                       void* h_out, void* d_out, uint64_t n, const void* init_host) {
    using A = typename ScanTypes<T>::A;
    constexpr int TILE = ScanShape<T>::TILE;
    const uint64_t tiles = (n + TILE - 1) / TILE;
    const bool bulk = (reinterpret_cast<uintptr_t>(d_in) % 16 == 0) &&
                      (reinterpret_cast<uintptr_t>(d_out) % 16 == 0);
    if (tiles > 0x7fffffffull || !bulk || !ws.copy_streams()) {
        cudaGetLastError();
        // one launch, copies before and after it
        cudaStream_t s = ws.stream();
        if (h_in && !arena_copy_async(const_cast<void*>(d_in), h_in, n * sizeof(T), true, s))
            return false;
        if (!scan_typed<T>(ws, exclusive, d_in, d_out, n, init_host)) return false;
        return !h_out || arena_copy_async(h_out, d_out, n * sizeof(T), false, s);
    }
    char* scratch = ws.scratch(tiles);
    if (!scratch) return false;
    auto ts = tile_status_at<A>(scratch, ws.next_epoch(), &ws.d_slot->spin_error);
    A init = A(0);
    if (exclusive && init_host) {
        T v;
        memcpy(&v, init_host, sizeof(T));
        init = (A)v;
    }
    const T* in = static_cast<const T*>(d_in);
    T* out = static_cast<T*>(d_out);
    cudaStream_t s = ws.stream();
    // On a failure part way, no copy may outlive the call: wait for both copy streams.
    auto fail = [&]() {
        cudaStreamSynchronize(ws.copy_up);
        cudaStreamSynchronize(ws.copy_down);
        cudaGetLastError();
        return false;
    };
    // the copy streams start after everything already queued on the workspace stream
    if (!cuda_ok(cudaEventRecord(ws.ev_copy[0], s), "copy event") ||
        !cuda_ok(cudaStreamWaitEvent(ws.copy_up, ws.ev_copy[0], 0), "copy wait") ||
        !cuda_ok(cudaStreamWaitEvent(ws.copy_down, ws.ev_copy[0], 0), "copy wait"))
        return fail();
    uint64_t chunks = 0;
    for (uint64_t t0 = 0; t0 < tiles; t0 += kCopyChunkTiles, ++chunks) {
        const uint64_t t1 = t0 + kCopyChunkTiles < tiles ? t0 + kCopyChunkTiles : tiles;
        const uint64_t e0 = t0 * TILE, e1 = t1 * TILE < n ? t1 * TILE : n;
        const size_t off = e0 * sizeof(T), bytes = (e1 - e0) * sizeof(T);
        if (h_in) {
            if (!arena_copy_async(const_cast<T*>(in) + e0, static_cast<const char*>(h_in) + off,
                                  bytes, true, ws.copy_up) ||
                !cuda_ok(cudaEventRecord(ws.ev_copy[1], ws.copy_up), "copy event") ||
                !cuda_ok(cudaStreamWaitEvent(s, ws.ev_copy[1], 0), "copy wait"))
                return fail();
        }
        uint32_t* counters = reinterpret_cast<uint32_t*>(scratch + ScratchOff::counters);
        const bool ok =
            exclusive ? launch_tiles_single<T, true, true>(in, out, n, init, ts, t1 - t0, s, t0, counters)
                      : launch_tiles_single<T, false, true>(in, out, n, init, ts, t1 - t0, s, t0, counters);
        if (!ok) return fail();
        if (h_out) {
            if (!cuda_ok(cudaEventRecord(ws.ev_copy[2], s), "copy event") ||
                !cuda_ok(cudaStreamWaitEvent(ws.copy_down, ws.ev_copy[2], 0), "copy wait") ||
                !arena_copy_async(static_cast<char*>(h_out) + off, out + e0, bytes, false,
                                  ws.copy_down))
                return fail();
        }
    }
    count_launch((unsigned)chunks);
    // the workspace stream (what a synchronous call waits on) ends after the last download
    if (!cuda_ok(cudaEventRecord(ws.ev_copy[3], ws.copy_down), "copy event") ||
        !cuda_ok(cudaStreamWaitEvent(s, ws.ev_copy[3], 0), "copy wait"))
        return fail();
    return cuda_ok(cudaGetLastError(), "k_scan launch");
}

}  // namespace

bool launch_scan_copies(Workspace& ws, DType t, bool exclusive, const void* h_in,
                        const void* d_in, void* h_out, void* d_out, size_t n,
                        const void* init_host) {
    switch (t) {
        case DType::F32:
            return scan_copies_typed<float>(ws, exclusive, h_in, d_in, h_out, d_out, n, init_host);
        case DType::F64:
            return scan_copies_typed<double>(ws, exclusive, h_in, d_in, h_out, d_out, n, init_host);
        case DType::I32:
            return scan_copies_typed<int32_t>(ws, exclusive, h_in, d_in, h_out, d_out, n, init_host);
        case DType::I64:
            return scan_copies_typed<int64_t>(ws, exclusive, h_in, d_in, h_out, d_out, n, init_host);
        case DType::U32:
            return scan_copies_typed<uint32_t>(ws, exclusive, h_in, d_in, h_out, d_out, n, init_host);
        case DType::U64:
            return scan_copies_typed<uint64_t>(ws, exclusive, h_in, d_in, h_out, d_out, n, init_host);
        default: break;
    }
    set_error(PARALLAX_ERR_INVALID_ARGUMENT, "scan: unsupported element type");
    return false;
}

bool launch_scan(Workspace& ws, DType t, bool exclusive, const void* d_in, void* d_out, size_t n,
                 const void* init_host) {
    switch (t) {
        case DType::F32: return scan_typed<float>(ws, exclusive, d_in, d_out, n, init_host);
        case DType::F64: return scan_typed<double>(ws, exclusive, d_in, d_out, n, init_host);
        case DType::I32: return scan_typed<int32_t>(ws, exclusive, d_in, d_out, n, init_host);
        case DType::I64: return scan_typed<int64_t>(ws, exclusive, d_in, d_out, n, init_host);
        case DType::U32: return scan_typed<uint32_t>(ws, exclusive, d_in, d_out, n, init_host);
        case DType::U64: return scan_typed<uint64_t>(ws, exclusive, d_in, d_out, n, init_host);
        default: break;
    }
    set_error(PARALLAX_ERR_INVALID_ARGUMENT, "scan: unsupported element type");
    return false;
}

// One scan tile launched as tile 1 of a fresh look-back epoch: tile 0 never publishes in
// that epoch, so the tile's look-back wait can only end by giving up after `polls` polls.
int check_bounded_wait(uint32_t polls) {
    using T = int32_t;
    using A = ScanTypes<T>::A;
    constexpr uint64_t TILE = ScanShape<T>::TILE;
    Workspace* ws = workspace();
    if (!ws) {
        set_error(PARALLAX_ERR_NO_DEVICE, "parallax_check_bounded_wait: no CUDA device");
        return PARALLAX_ERR_NO_DEVICE;
    }
    char* scratch = ws->scratch(2);
    T* buf = static_cast<T*>(ws->temp(2 * TILE * sizeof(T) * 2));
    if (!scratch || !buf) return last_error();
    cudaStream_t s = ws->stream();
    if (!cuda_ok(cudaMemsetAsync(buf, 0, 2 * TILE * sizeof(T), s), "check_bounded_wait: input"))
        return PARALLAX_ERR_CUDA;
    auto ts = tile_status_at<A>(scratch, ws->next_epoch(), &ws->d_slot->spin_error);
    ts.limit = polls;
    if (!launch_tiles_single<T, false, true>(buf, buf + 2 * TILE, 2 * TILE, A(0), ts, 1, s, 1))
        return last_error() ? last_error() : PARALLAX_ERR_CUDA;
    count_launch();
    return sync_stream(*ws);
}

}  // namespace pxb

PXB_EXPORT int parallax_check_bounded_wait(uint32_t polls) {
    pxb::set_ok();
    if (polls == 0 || polls > pxb::kSpinLimit) {
        pxb::set_error(PARALLAX_ERR_INVALID_ARGUMENT,
                       "parallax_check_bounded_wait: polls must be in [1, %u]", pxb::kSpinLimit);
        return PARALLAX_ERR_INVALID_ARGUMENT;
    }
    return pxb::check_bounded_wait(polls);
}

// ---- allocation-free scan -----------------------------------------------------------------
// Some callers cannot allocate device memory at all: code that runs inside an allocation
// hook (a malloc / operator new interposer that routes the heap into the arena would
// re-enter itself if the runtime allocated), or a process whose device memory has been
// handed to its own pool. parallax_scan_noalloc gives them the single-pass scan with no
// allocation by the runtime: the look-back status lives in the fixed static device array
// below (384.25 KiB, held on every GPU that loads this library until the process exits),
// the caller passes device buffers for input and output and a stream, and no workspace,
// stream, event or pinned slot is created.
namespace pxb {
namespace {

constexpr uint64_t kNoAllocTiles = 24576;  // look-back status entries
constexpr size_t kNoAllocBytes = 256 + kNoAllocTiles * sizeof(StatusEntry);
// [0, 4): in-kernel wait-timeout code; [256, ...): look-back status entries. Static device
// memory starts zeroed; later calls find stale entries from older epochs, which read as
// "not ready", so only the timeout code is cleared per call.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

constexpr int kNoAllocMaxDevices = 64;
struct NoAllocDevice {
    bool ready = false;
    char* scratch = nullptr;  // device address of g_noalloc_scratch on that device
    uint32_t epoch = 0;
};
std::mutex g_noalloc_mu;
NoAllocDevice g_noalloc[kNoAllocMaxDevices];

template <typename T>
uint64_t noalloc_max_elements() {
    return kNoAllocTiles * (uint64_t)ScanShape<T>::TILE;
}

template <typename T>
bool noalloc_launch(const void* d_in, void* d_out, uint64_t n, const void* init_host,
                    cudaStream_t s, char* scratch, uint32_t epoch) {
    using A = typename ScanTypes<T>::A;
    constexpr int TILE = ScanShape<T>::TILE;
    const uint64_t tiles = (n + TILE - 1) / TILE;
    TileStatus<A> ts;
    ts.e = reinterpret_cast<StatusEntry*>(scratch + 256);
    ts.epoch = epoch;
    ts.err = reinterpret_cast<int32_t*>(scratch);
    A init = A(0);
    if (init_host) {
        T v;
        memcpy(&v, init_host, sizeof(T));
        init = (A)v;
    }
    const bool bulk = (reinterpret_cast<uintptr_t>(d_in) % 16 == 0) &&
                      (reinterpret_cast<uintptr_t>(d_out) % 16 == 0);
    const T* in = static_cast<const T*>(d_in);
    T* out = static_cast<T*>(d_out);
    bool ok;
    if (init_host) {
        ok = bulk ? launch_tiles_single<T, true, true>(in, out, n, init, ts, tiles, s)
                  : launch_tiles_single<T, true, false>(in, out, n, init, ts, tiles, s);
    } else {
        ok = bulk ? launch_tiles_single<T, false, true>(in, out, n, init, ts, tiles, s)
                  : launch_tiles_single<T, false, false>(in, out, n, init, ts, tiles, s);
    }
    if (!ok) return false;
    count_launch();
    return cuda_ok(cudaGetLastError(), "parallax_scan_noalloc launch");
}

}  // namespace
}  // namespace pxb

using namespace pxb;

PXB_EXPORT int parallax_scan_noalloc(parallax_kernel_t scan_kernel, const void* input,
                                     void* output, size_t count, size_t elem_size,
                                     const void* init, void* cuda_stream) {
    set_ok();
    Handle* h = as_handle(scan_kernel);
    if (!h || h->kind != Kind::SCAN) {
        set_error(PARALLAX_ERR_INVALID_HANDLE, "parallax_scan_noalloc: not a scan kernel handle");
        return PARALLAX_ERR_INVALID_HANDLE;
    }
    if (dtype_size(h->dtype) != elem_size || !input || !output) {
        set_error(PARALLAX_ERR_INVALID_ARGUMENT,
                  "parallax_scan_noalloc: null buffer or elem_size %zu does not match the handle",
                  elem_size);
        return PARALLAX_ERR_INVALID_ARGUMENT;
    }
    if (count == 0) return PARALLAX_OK;
    uint64_t max_n = 0;
    switch (h->dtype) {
        case DType::F32: max_n = noalloc_max_elements<float>(); break;
        case DType::F64: max_n = noalloc_max_elements<double>(); break;
        case DType::I32: max_n = noalloc_max_elements<int32_t>(); break;
        case DType::I64: max_n = noalloc_max_elements<int64_t>(); break;
        case DType::U32: max_n = noalloc_max_elements<uint32_t>(); break;
        case DType::U64: max_n = noalloc_max_elements<uint64_t>(); break;
        default: break;
    }
    if (count > max_n) {
        set_error(PARALLAX_ERR_INVALID_ARGUMENT,
                  "parallax_scan_noalloc: %zu elements exceed its maximum of %llu for this "
                  "element type (%llu look-back tiles in a %zu-byte static array); use "
                  "parallax_scan or parallax_exclusive_scan",
                  count, (unsigned long long)max_n, (unsigned long long)kNoAllocTiles,
                  kNoAllocBytes);
        return PARALLAX_ERR_INVALID_ARGUMENT;
    }
    int dev = 0;
    if (!cuda_ok(cudaGetDevice(&dev), "parallax_scan_noalloc: cudaGetDevice"))
        return PARALLAX_ERR_CUDA;
    if (dev < 0 || dev >= kNoAllocMaxDevices) {
        set_error(PARALLAX_ERR_UNSUPPORTED, "parallax_scan_noalloc: device %d out of range", dev);
        return PARALLAX_ERR_UNSUPPORTED;
    }
    cudaStream_t s = static_cast<cudaStream_t>(cuda_stream);
    char* scratch = nullptr;
    uint32_t epoch = 0;
    {
        std::lock_guard<std::mutex> g(g_noalloc_mu);
        NoAllocDevice& d = g_noalloc[dev];
        if (!d.ready) {
            // Once per device, with that device current. The name of a __device__ array is
            // a host-side stand-in in host code; only this address reaches the kernel.
            void* p = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess || !p) {
                cuda_ok(e == cudaSuccess ? cudaErrorInvalidSymbol : e,
                        "parallax_scan_noalloc: cudaGetSymbolAddress");
                return PARALLAX_ERR_CUDA;
            }
            d.scratch = static_cast<char*>(p);
            d.epoch = 0;
            d.ready = true;
        }
        if (++d.epoch >= (1u << 30)) {  // epoch wrap: stale words could alias, clear them
            if (!cuda_ok(cudaMemsetAsync(d.scratch + 256, 0, kNoAllocBytes - 256, s),
                         "parallax_scan_noalloc: clear status"))
                return PARALLAX_ERR_CUDA;
            d.epoch = 1;
        }
        scratch = d.scratch;
        epoch = d.epoch;
    }
    if (!cuda_ok(cudaMemsetAsync(scratch, 0, sizeof(int32_t), s),
                 "parallax_scan_noalloc: clear timeout code"))
        return PARALLAX_ERR_CUDA;
    bool ok = false;
    switch (h->dtype) {
        case DType::F32: ok = noalloc_launch<float>(input, output, count, init, s, scratch, epoch); break;
        case DType::F64: ok = noalloc_launch<double>(input, output, count, init, s, scratch, epoch); break;
        case DType::I32: ok = noalloc_launch<int32_t>(input, output, count, init, s, scratch, epoch); break;
        case DType::I64: ok = noalloc_launch<int64_t>(input, output, count, init, s, scratch, epoch); break;
        case DType::U32: ok = noalloc_launch<uint32_t>(input, output, count, init, s, scratch, epoch); break;
        case DType::U64: ok = noalloc_launch<uint64_t>(input, output, count, init, s, scratch, epoch); break;
        default: break;
    }
    if (!ok) return PARALLAX_ERR_CUDA;
    int32_t code = 0;
    if (!cuda_ok(cudaMemcpyAsync(&code, scratch, sizeof code, cudaMemcpyDeviceToHost, s),
                 "parallax_scan_noalloc: read timeout code") ||
        !cuda_ok(cudaStreamSynchronize(s), "parallax_scan_noalloc: stream synchronize"))
        return PARALLAX_ERR_CUDA;
    if (code) {
        set_error(PARALLAX_ERR_DEVICE_SPIN, "parallax_scan_noalloc: in-kernel wait gave up (%d)",
                  code);
        return PARALLAX_ERR_DEVICE_SPIN;
    }
    return PARALLAX_OK;
}
