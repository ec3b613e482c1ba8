// Stable single-pass compaction: copy_if / remove_if / unique, and stable partition.
//
// Reference: four or more dispatches with fence waits - a flags kernel writing 1.0/0.0
// in the ELEMENT type, a multi-pass scan of those flags, a host read of the last
// position, then a scatter kernel (src/kernel/kernel_launcher.cpp:1701-1791,
// shaders/flags.comp:14-18, shaders/scatter.comp:15-22). Element-typed positions make
// fp32 counts inexact beyond 2^24; here counts are 32-bit within a tile and 64-bit
// across tiles.
//
// Here: one 512-thread CTA per 112 KiB tile (two per SM), in blockIdx order, staged as two
// bulk-copied sub-tiles (tiles.cuh). Phase 1 evaluates the predicate (or the adjacent-difference test for
// unique) on 28 / 14 consecutive elements per thread as each sub-tile lands, keeps the
// flags as bit masks, and ranks the kept elements with one shuffle scan per sub-tile and
// one 32-lane scan over the (sub-tile, warp) counts; warp 0 gets the tile's output offset
// by decoupled look-back on kept counts. Phase 2 packs the kept elements at the front of
// the staged tile, sub-tile by sub-tile (a packed element never lands beyond the sub-tile
// being packed), and writes them with coalesced stores. Traffic: n*s read + k*s written.
// Partition writes every element: kept ones to [0, k), the rest in order to [k, n). The
// rejected elements' offsets need k, so partition runs a count pass first (one read of
// the input); each sub-tile is then permuted in shared memory (kept run, rejected run)
// and both runs are written with coalesced stores.
#include <stdint.h>

#include <type_traits>

#include "../lookback.cuh"
#include "../runtime.hpp"
#include "../tiles.cuh"
#include "../tma.cuh"

namespace pxb {
namespace {

// Tile shape (measured: 112 KiB tiles, 2 CTAs/SM); can be overridden at build time
// (PXB_COMPACT_BLOCK / _VPT / _SUB / _CTAS) to sweep it; kSub x (kBlock / 32) must be 32.
#ifndef PXB_COMPACT_BLOCK
#define PXB_COMPACT_BLOCK 512
#endif
#ifndef PXB_COMPACT_VPT
#define PXB_COMPACT_VPT 7
#endif
#ifndef PXB_COMPACT_SUB
#define PXB_COMPACT_SUB 2
#endif
#ifndef PXB_COMPACT_CTAS
#define PXB_COMPACT_CTAS 2
#endif
constexpr int kBlock = PXB_COMPACT_BLOCK;
constexpr int kVpt = PXB_COMPACT_VPT;
constexpr int kSub = PXB_COMPACT_SUB;
constexpr int kCtasPerSm = PXB_COMPACT_CTAS;

template <typename T>
struct Shape {
    static constexpr int V = 16 / sizeof(T);
    static constexpr int ITEMS = kVpt * V;
    static constexpr int SUB = kBlock * ITEMS;
    static constexpr int TILE = kSub * SUB;
    static constexpr size_t SMEM = TILE * sizeof(T);
};

template <typename T>
struct PredDev {
    PredKind kind;
    bool negate;
    T c, m, r;
    FastMod32 fm;           // 32-bit element types: m as an invariant divisor
    const uint8_t* fl;      // FLAGS: one byte per element, written by a registered image
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
                if constexpr (std::is_integral<T>::value) v = x % m == r;
                else v = false;
                break;
            default: v = false; break;
        }
        return v != negate;
    }
    // Flag bits of one row whose first element has global index gi: the switch on the
    // (CTA-uniform) kind is taken once per row.
    template <int ITEMS>
    __device__ __forceinline__ uint32_t flags(const T (&x)[ITEMS], uint64_t gi) const {
        uint32_t f = 0;
        switch (kind) {
            case PredKind::FLAGS:
                // rows start at multiples of ITEMS (28 or 14), so the row's flag bytes are
                // 4-byte (or 2-byte) aligned; the array is padded past the last tile
                if constexpr (ITEMS % 4 == 0) {
                    const uint32_t* w = reinterpret_cast<const uint32_t*>(fl + gi);
#pragma unroll
                    for (int v = 0; v < ITEMS / 4; ++v) {
                        const uint32_t b = __ldg(w + v);
#pragma unroll
                        for (int k = 0; k < 4; ++k)
                            f |= (uint32_t)((((b >> (8 * k)) & 0xffu) != 0u) != negate) << (4 * v + k);
                    }
                } else {
                    static_assert(ITEMS % 2 == 0, "rows of an even number of elements");
                    const uint16_t* w = reinterpret_cast<const uint16_t*>(fl + gi);
#pragma unroll
                    for (int v = 0; v < ITEMS / 2; ++v) {
                        const uint32_t b = __ldg(w + v);
#pragma unroll
                        for (int k = 0; k < 2; ++k)
                            f |= (uint32_t)((((b >> (8 * k)) & 0xffu) != 0u) != negate) << (2 * v + k);
                    }
                }
                break;
#define PXB_ROW(KIND, EXPR)                                              \
            case PredKind::KIND:                                          \
                _Pragma("unroll") for (int j = 0; j < ITEMS; ++j)          \
                    f |= (uint32_t)((EXPR) != negate) << j;                \
                break;
            PXB_ROW(GT, x[j] > c)
            PXB_ROW(GE, x[j] >= c)
            PXB_ROW(LT, x[j] < c)
            PXB_ROW(LE, x[j] <= c)
            PXB_ROW(EQ, x[j] == c)
            PXB_ROW(NE, x[j] != c)
            PXB_ROW(NONZERO, x[j] != T(0))
            case PredKind::MOD:
                if constexpr (std::is_integral<T>::value && sizeof(T) == 4) {
                    if (r == T(0)) {  // divisibility: a multiply and a compare per element
#pragma unroll
                        for (int j = 0; j < ITEMS; ++j) f |= (uint32_t)(fm.eq0(x[j]) != negate) << j;
                        break;
                    }
                }
#pragma unroll
                for (int j = 0; j < ITEMS; ++j) f |= (uint32_t)(mod_eq(x[j]) != negate) << j;
                break;
#undef PXB_ROW
            default: break;
        }
        return f;
    }
    // x % m == r with C semantics; 32-bit integers divide by the precomputed invariant
    // divisor instead of the long division.
    __device__ __forceinline__ bool mod_eq(T x) const {
        if constexpr (std::is_integral<T>::value && sizeof(T) == 4) {
            return fm.eq(x, r);
        } else if constexpr (std::is_integral<T>::value) {  // x % -1 == 0, no overflow
            return (std::is_signed<T>::value && m == T(-1)) ? r == T(0) : x % m == r;
        } else {
            return false;
        }
    }
};

template <typename T, int ITEMS, int V>
__device__ __forceinline__ void load_row(const T* row_ptr, T (&x)[ITEMS]) {
    const uint4* row = reinterpret_cast<const uint4*>(row_ptr);
#pragma unroll
    for (int v = 0; v < ITEMS / V; ++v) {
        const uint4 r = row[v];
        const T* e = reinterpret_cast<const T*>(&r);
#pragma unroll
        for (int k = 0; k < V; ++k) x[v * V + k] = e[k];
    }
}

// Shared state of one CTA's tile processing.
struct CompactSmem {
    uint32_t cnt[32];               // (sub-tile, warp) kept counts
    uint64_t red[kBlock / 32 + 1];  // look-back scratch
    int first[kBlock / 32];
};

// One staged tile: flags, ranks, look-back, then packed (select / unique) or scattered
// (partition) output. MODE: 0 select (copy_if / remove_if), 1 unique, 2 partition.
// `prev_of_tile` is the element before the tile (unique only). Ends with a barrier after
// which the tile buffer may be refilled.
template <typename T, int MODE, bool BULK>
__device__ __forceinline__ void compact_tile(T* buf, uint64_t* bars, uint32_t parity,
                                             CompactSmem& sm, uint64_t tile, uint64_t base,
                                             uint32_t cnt, T prev_of_tile, T* out, uint64_t n,
                                             const PredDev<T>& pred,
                                             const TileStatus<uint64_t>& ts,
                                             const unsigned long long* num_true,
                                             unsigned long long* count_out, bool last_tile) {
    constexpr int V = Shape<T>::V;
    constexpr int ITEMS = Shape<T>::ITEMS;
    constexpr int SUB = Shape<T>::SUB;
    constexpr int WARPS = kBlock / 32;
    static_assert(kSub * WARPS == 32, "one lane per (sub-tile, warp)");
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t row0 = (uint32_t)tid * ITEMS;

    // ---- phase 1: flags and ranks ----
    uint32_t fl[kSub];   // bit j: element j of this thread's row in sub-tile s is kept
    uint32_t tex[kSub];  // kept elements before this row within its warp
#pragma unroll
    for (int s = 0; s < kSub; ++s) {
        if constexpr (BULK) wait_bar(&bars[s], parity, ts.err);
        const uint32_t e0 = (uint32_t)s * SUB + row0;  // tile index of the row's first element
        T x[ITEMS];
        load_row<T, ITEMS, V>(buf + e0, x);
        uint32_t f = 0;
        if constexpr (MODE == 1) {
            const T prev = e0 > 0 ? buf[e0 - 1] : prev_of_tile;
            const bool first_global = base == 0 && e0 == 0;
#pragma unroll
            for (int j = 0; j < ITEMS; ++j) {
                const bool keep = (j == 0 && first_global) || !(x[j] == (j ? x[j - 1] : prev));
                if (e0 + j < cnt && keep) f |= 1u << j;
            }
        } else {
            f = pred.template flags<ITEMS>(x, base + e0);
            if (e0 + ITEMS > cnt) f &= e0 >= cnt ? 0u : (1u << (cnt - e0)) - 1u;
        }
        fl[s] = f;
        const uint32_t incl = warp_inclusive_scan((uint32_t)__popc(f), OpSum());
        const uint32_t ex = shfl_up(incl, 1);
        tex[s] = lane == 0 ? 0u : ex;
        if (lane == 31) sm.cnt[s * WARPS + warp] = incl;
    }
    __syncthreads();
    // Every warp scans the 32 (sub-tile, warp) counts itself, then the whole CTA runs the
    // look-back on kept counts.
    uint32_t woff[kSub];  // kept elements before this warp's rows within the tile
    uint32_t tile_kept;
    {
        const uint32_t v = sm.cnt[lane];
        const uint32_t vi = warp_inclusive_scan(v, OpSum());
        tile_kept = shfl_idx(vi, 31);
        uint32_t vex = shfl_up(vi, 1);
        if (lane == 0) vex = 0;
#pragma unroll
        for (int s = 0; s < kSub; ++s) woff[s] = shfl_idx(vex, s * WARPS + warp);
    }
    const uint64_t prefix =
        lookback_cta<uint64_t, kBlock, true>(ts, tile, (uint64_t)tile_kept, sm.red, sm.first);
    if (MODE != 2 && last_tile && tid == 0) *count_out = prefix + tile_kept;

    if constexpr (MODE == 2) {
        // ---- partition: per sub-tile, kept elements are packed at its front and the
        // rejected ones after them (an in-place permutation of the sub-tile, done from
        // registers after a barrier), then both runs are stored with coalesced writes:
        // kept to [prefix + kept before the sub-tile, ...), rejected to
        // [num_true + rejected before the sub-tile, ...).
        const uint64_t nt = *num_true;
        const uint64_t rej_base = nt + (base - prefix);
        uint32_t sub_before[kSub + 1];  // kept elements of the tile before each sub-tile
        {
            const uint32_t v = sm.cnt[lane];
            const uint32_t vi = warp_inclusive_scan(v, OpSum());
            uint32_t vex = shfl_up(vi, 1);
            if (lane == 0) vex = 0;
#pragma unroll
            for (int s = 0; s < kSub; ++s) sub_before[s] = shfl_idx(vex, s * WARPS);
            sub_before[kSub] = tile_kept;
        }
#pragma unroll
        for (int s = 0; s < kSub; ++s) {
            const uint32_t s0 = (uint32_t)s * SUB;
            const uint32_t ks = sub_before[s + 1] - sub_before[s];      // kept in sub-tile
            const uint32_t valid = cnt > s0 ? (cnt - s0 < (uint32_t)SUB ? cnt - s0 : (uint32_t)SUB) : 0u;
            T* sb = buf + s0;
            T x[ITEMS];
            load_row<T, ITEMS, V>(sb + row0, x);
            __syncthreads();  // every row of sub-tile s is in registers before permuting
            uint32_t rk = woff[s] + tex[s] - sub_before[s];  // kept before this row (sub-tile)
            uint32_t rr = row0 - rk;                          // rejected before this row
#pragma unroll
            for (int j = 0; j < ITEMS; ++j) {
                if (row0 + j >= valid) break;
                if (fl[s] >> j & 1u) sb[rk++] = x[j];
                else sb[ks + rr++] = x[j];
            }
            __syncthreads();
            const uint64_t kdst = prefix + sub_before[s];
            const uint64_t rdst = rej_base + (s0 - sub_before[s]);
            for (uint32_t i = tid; i < valid; i += kBlock) {
                const uint64_t dst = i < ks ? kdst + i : rdst + (i - ks);
                if (dst < n) out[dst] = sb[i];
                else *ts.err = 3;  // only reachable after a failed wait: never write out of range
            }
        }
        if (tid == 0 && last_tile) *count_out = nt;
    } else {
        // ---- pack kept elements at the front of the tile, then store them ----
#pragma unroll
        for (int s = 0; s < kSub; ++s) {
            T x[ITEMS];
            load_row<T, ITEMS, V>(buf + (uint32_t)s * SUB + row0, x);
            __syncthreads();  // every row of sub-tile s is in registers before packing
            uint32_t r = woff[s] + tex[s];
#pragma unroll
            for (int j = 0; j < ITEMS; ++j)
                if (fl[s] >> j & 1u) buf[r++] = x[j];
        }
        __syncthreads();
        for (uint32_t i = tid; i < tile_kept; i += kBlock) {
            if (prefix + i < n) out[prefix + i] = buf[i];
            else *ts.err = 3;
        }
    }
    __syncthreads();  // buffer and shared state free for the next tile
}

// One CTA per tile, in blockIdx order, or in the order of an atomic claim counter when
// `claim` is given (see tile_claim()).
template <typename T, int MODE, bool BULK>
__global__ void __launch_bounds__(kBlock, kCtasPerSm)
k_compact(const T* in, T* out, uint64_t n, PredDev<T> pred, TileStatus<uint64_t> ts,
          const unsigned long long* __restrict__ num_true,
          unsigned long long* __restrict__ count_out, uint32_t* claim) {
    constexpr int SUB = Shape<T>::SUB;
    constexpr int TILE = Shape<T>::TILE;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    T* buf = reinterpret_cast<T*>(smem_raw);
    __shared__ __align__(8) uint64_t bars[kSub];
    __shared__ CompactSmem sm;
    __shared__ uint32_t s_claim;
    const uint64_t tile = claim ? tile_claim(claim, s_claim) : blockIdx.x;
    const uint64_t base = tile * (uint64_t)TILE;
    const uint64_t rem = n - base;
    const uint32_t cnt = rem < (uint64_t)TILE ? (uint32_t)rem : (uint32_t)TILE;
    stage_tile<T, SUB, kSub, kBlock, BULK>(buf, bars, in, base, cnt);
    const T prev = (MODE == 1 && base > 0) ? in[base - 1] : T(0);
    __syncthreads();
    compact_tile<T, MODE, BULK>(buf, bars, 0, sm, tile, base, cnt, prev, out, n, pred, ts,
                                num_true, count_out, tile == gridDim.x - 1);
    if (claim && threadIdx.x == 0) persistent_exit(claim);
}

// Persistent CTAs (two per SM), two tile buffers each: the next claimed tile's bulk copies
// are in flight while the current tile is compacted. Input 16-byte aligned.
template <typename T, int MODE>
__global__ void __launch_bounds__(kBlock, 2)
k_compact_persistent(const T* in, T* out, uint64_t n, uint64_t num_tiles, PredDev<T> pred,
                     TileStatus<uint64_t> ts, const unsigned long long* __restrict__ num_true,
                     unsigned long long* __restrict__ count_out, uint32_t* counters) {
    constexpr int SUB = Shape<T>::SUB;
    constexpr int TILE = Shape<T>::TILE;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    T* const buf0 = reinterpret_cast<T*>(smem_raw);  // buffer b at buf0 + b * TILE
    __shared__ __align__(8) uint64_t bars[2][kSub];
    __shared__ CompactSmem sm;
    __shared__ uint32_t s_tile[2];
    __shared__ T s_prev[2];
    const int tid = threadIdx.x;

    auto claim_and_issue = [&](int b) {  // thread 0 only
        const uint32_t t = atomicAdd(&counters[0], 1u);
        s_tile[b] = t;
        if (t < num_tiles) {
            const uint64_t base = (uint64_t)t * TILE;
            const uint64_t rem = n - base;
            issue_tile<T, SUB, kSub>(buf0 + (size_t)b * TILE, bars[b], in, base,
                                     rem < (uint64_t)TILE ? (uint32_t)rem : (uint32_t)TILE);
            // the element before the tile (unique): its latency hides behind this round
            s_prev[b] = (MODE == 1 && base > 0) ? in[base - 1] : T(0);
        }
    };
    if (tid == 0) {
#pragma unroll
        for (int b = 0; b < 2; ++b)
#pragma unroll
            for (int s = 0; s < kSub; ++s) mbar_init(&bars[b][s], 1);
        fence_mbar_init();
        claim_and_issue(0);
    }
    __syncthreads();
    for (uint32_t it = 0;; ++it) {
        const int b = it & 1;
        const uint32_t parity = (it >> 1) & 1u;
        const uint32_t cur = s_tile[b];
        if (cur >= num_tiles) break;
        const T prev = s_prev[b];
        if (tid == 0) {
            fence_proxy_async_smem();
            claim_and_issue(b ^ 1);
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
        compact_tile<T, MODE, true>(buf, bars[b], parity, sm, cur, base, cnt, prev, out, n,
                                    pred, ts, num_true, count_out, cur == num_tiles - 1);
    }
    if (tid == 0) persistent_exit(counters);
}

template <typename T>
PredDev<T> make_pred(const Pred& p) {
    PredDev<T> e;
    e.kind = p.kind;
    e.negate = p.negate;
    if (std::is_floating_point<T>::value) e.c = (T)p.f;
    else if (std::is_signed<T>::value) e.c = (T)p.i;
    else e.c = (T)p.u;
    e.m = (T)p.mod_m;
    e.r = (T)p.mod_r;
    if (std::is_integral<T>::value && sizeof(T) == 4) e.fm = FastMod32::make((int64_t)e.m);
    e.fl = p.flags;
    return e;
}

template <typename T, int MODE>
bool launch_mode(uint64_t tiles, cudaStream_t s, bool bulk, const T* in, T* out, uint64_t n,
                 PredDev<T> p, TileStatus<uint64_t> ts, const unsigned long long* nt,
                 unsigned long long* count_out, uint32_t* counters) {
    static const bool persistent = getenv("PARALLAX_PERSISTENT_TILES") != nullptr;
    if (bulk && !persistent) {
        if (!smem_opt_in<k_compact<T, MODE, true>>(Shape<T>::SMEM))
            return cuda_ok(cudaGetLastError(), "k_compact shared-memory opt-in");
        k_compact<T, MODE, true><<<(unsigned)tiles, kBlock, Shape<T>::SMEM, s>>>(
            in, out, n, p, ts, nt, count_out, PXB_TILE_CLAIM ? counters : nullptr);
        return true;
    }
    if (bulk) {
        constexpr size_t smem = 2 * Shape<T>::SMEM;
        if (!smem_opt_in<k_compact_persistent<T, MODE>>(smem))
            return cuda_ok(cudaGetLastError(), "k_compact_persistent shared-memory opt-in");
        uint64_t grid = 2ull * device_info().sm_count;
        if (grid > tiles) grid = tiles;
        k_compact_persistent<T, MODE><<<(unsigned)grid, kBlock, smem, s>>>(
            in, out, n, tiles, p, ts, nt, count_out, counters);
        return true;
    }
    if (!smem_opt_in<k_compact<T, MODE, false>>(Shape<T>::SMEM))
        return cuda_ok(cudaGetLastError(), "k_compact shared-memory opt-in");
    k_compact<T, MODE, false><<<(unsigned)tiles, kBlock, Shape<T>::SMEM, s>>>(
        in, out, n, p, ts, nt, count_out, PXB_TILE_CLAIM ? counters : nullptr);
    return true;
}

template <typename T>
bool compact_typed(Workspace& ws, CompactMode mode, const Pred& pr, const void* d_in,
                   void* d_out, uint64_t n, uint64_t* d_count) {
    constexpr int TILE = Shape<T>::TILE;
    const uint64_t tiles = (n + TILE - 1) / TILE;
    if (tiles > 0x7fffffffull) {
        set_error(PARALLAX_ERR_INVALID_ARGUMENT, "compaction: too many elements");
        return false;
    }
    char* scratch = ws.scratch(tiles);
    if (!scratch) return false;
    auto* nt = reinterpret_cast<unsigned long long*>(scratch + ScratchOff::num_true);
    if (pr.kind == PredKind::FLAGS && (!pr.flags || reinterpret_cast<uintptr_t>(pr.flags) % 4)) {
        set_error(PARALLAX_ERR_INVALID_ARGUMENT, "compaction: flags array missing or unaligned");
        return false;
    }
    if (mode == CompactMode::PARTITION) {
        // count pass: k = |{i : pred(in[i])}| into device scratch
        const bool ok = pr.kind == PredKind::FLAGS
            ? launch_count_flags(ws, pr.flags, n, reinterpret_cast<uint64_t*>(nt))
            : launch_count_if(ws, dtype_of<T>(), pr, d_in, n, reinterpret_cast<uint64_t*>(nt));
        if (!ok) return false;
    }
    auto ts = tile_status_at<uint64_t>(scratch, ws.next_epoch(), &ws.d_slot->spin_error);
    // bulk copies only from HBM; the page-locked host mirror (small coherent operands,
    // whole-heap capture) takes plain loads
    const bool bulk = reinterpret_cast<uintptr_t>(d_in) % 16 == 0 && !arena_contains(d_in);
    const T* in = static_cast<const T*>(d_in);
    T* out = static_cast<T*>(d_out);
    auto* cnt_out = reinterpret_cast<unsigned long long*>(d_count);
    PredDev<T> p = make_pred<T>(pr);
    uint32_t* counters = reinterpret_cast<uint32_t*>(scratch + ScratchOff::counters);
    cudaStream_t s = ws.stream();
    // profile bytes: input read (+ the kept elements written, known only on the device)
    ProfScope prof(ws, mode == CompactMode::PARTITION ? "k_partition"
                       : mode == CompactMode::UNIQUE ? "k_unique" : "k_copy_if",
                   (mode == CompactMode::PARTITION ? 2 : 1) * n * sizeof(T));
    bool ok = false;
    switch (mode) {
        case CompactMode::SELECT:
            ok = launch_mode<T, 0>(tiles, s, bulk, in, out, n, p, ts, nt, cnt_out, counters);
            break;
        case CompactMode::UNIQUE:
            ok = launch_mode<T, 1>(tiles, s, bulk, in, out, n, p, ts, nt, cnt_out, counters);
            break;
        case CompactMode::PARTITION:
            ok = launch_mode<T, 2>(tiles, s, bulk, in, out, n, p, ts, nt, cnt_out, counters);
            break;
    }
    if (!ok) return false;
    count_launch();
    return cuda_ok(cudaGetLastError(), "k_compact launch");
}

}  // namespace

size_t compact_flags_padding(size_t n) {
    constexpr size_t kTile = Shape<uint32_t>::TILE;  // the largest tile, in elements
    static_assert(Shape<uint32_t>::TILE % Shape<uint64_t>::TILE == 0, "tile sizes nest");
    return (n + kTile - 1) / kTile * kTile + 16;
}

bool launch_compact(Workspace& ws, DType t, CompactMode mode, const Pred& p, const void* d_in,
                    void* d_out, size_t n, uint64_t* d_count) {
    switch (t) {
        case DType::F32: return compact_typed<float>(ws, mode, p, d_in, d_out, n, d_count);
        case DType::F64: return compact_typed<double>(ws, mode, p, d_in, d_out, n, d_count);
        case DType::I32: return compact_typed<int32_t>(ws, mode, p, d_in, d_out, n, d_count);
        case DType::I64: return compact_typed<int64_t>(ws, mode, p, d_in, d_out, n, d_count);
        case DType::U32: return compact_typed<uint32_t>(ws, mode, p, d_in, d_out, n, d_count);
        case DType::U64: return compact_typed<uint64_t>(ws, mode, p, d_in, d_out, n, d_count);
        default: break;
    }
    set_error(PARALLAX_ERR_INVALID_ARGUMENT, "compaction: unsupported element type");
    return false;
}

}  // namespace pxb
