// Stable single-pass compaction: copy_if / remove_if / unique, and stable partition.
//
// Reference: four or more dispatches with fence waits - a flags kernel writing 1.0/0.0
// in the ELEMENT type, a multi-pass scan of those flags, a host read of the last
// position, then a scatter kernel (src/kernel/kernel_launcher.cpp:1701-1791,
// shaders/flags.comp:14-18, shaders/scatter.comp:15-22). Element-typed positions make
// fp32 counts inexact beyond 2^24; here counts are 32-bit within a tile and 64-bit
// across tiles.
//
// Here: one CTA per tile, in blockIdx order. A CTA stages its tile with one bulk copy,
// evaluates the predicate (or the adjacent-difference test for unique) on 12 / 6
// consecutive elements per thread, ranks the kept elements with shuffle scans, gets the
// tile's output offset by decoupled look-back on kept counts, packs the kept elements in
// shared memory and writes them out with coalesced stores. Traffic: n*s read + k*s
// written.
// Partition writes every element: kept ones to [0, k), the rest in order to [k, n). The
// rejected elements' offsets need k, so partition runs a count pass first (one read of
// the input) and then the same kernel with two output cursors.
#include <stdint.h>

#include <type_traits>

#include "../lookback.cuh"
#include "../runtime.hpp"
#include "../tma.cuh"

namespace pxb {
namespace {

constexpr int kBlock = 256;
constexpr int kVpt = 3;

template <typename T>
struct Shape {
    static constexpr int V = 16 / sizeof(T);
    static constexpr int ITEMS = kVpt * V;
    static constexpr int TILE = kBlock * ITEMS;
};

template <typename T>
struct PredDev {
    PredKind kind;
    bool negate;
    T c, m, r;
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
};

// MODE: 0 select (copy_if / remove_if), 1 unique, 2 partition
template <typename T, int MODE, bool BULK>
__global__ void __launch_bounds__(kBlock)
k_compact(const T* in, T* out, uint64_t n, PredDev<T> pred,
          TileStatus<uint64_t> ts, const unsigned long long* __restrict__ num_true,
          unsigned long long* __restrict__ count_out) {
    constexpr int V = Shape<T>::V;
    constexpr int ITEMS = Shape<T>::ITEMS;
    constexpr int TILE = Shape<T>::TILE;
    __shared__ __align__(128) T buf[TILE];
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t s_warp[kBlock / 32];
    __shared__ uint32_t s_wex[kBlock / 32];
    __shared__ uint32_t s_kept;
    __shared__ uint64_t s_prefix;

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint64_t tile = blockIdx.x;
    const uint64_t base = tile * (uint64_t)TILE;
    const uint64_t rem = n - base;
    const uint32_t cnt = rem < (uint64_t)TILE ? (uint32_t)rem : (uint32_t)TILE;

    uint32_t bulk = 0;
    if constexpr (BULK) {
        bulk = (uint32_t)((cnt * sizeof(T)) / 16 * 16 / sizeof(T));
        if (tid == 0) {
            mbar_init(&bar, 1);
            fence_mbar_init();
            mbar_arrive_expect_tx(&bar, bulk * (uint32_t)sizeof(T));
            if (bulk) bulk_load(buf, in + base, bulk * (uint32_t)sizeof(T), &bar);
        }
    }
    for (uint32_t e = bulk + tid; e < (uint32_t)TILE; e += kBlock)
        buf[e] = e < cnt ? in[base + e] : T(0);
    T prev_of_tile = T(0);
    if (MODE == 1 && tid == 0 && base > 0) prev_of_tile = in[base - 1];
    __syncthreads();
    if constexpr (BULK) {
        uint32_t spins = 0;
        while (!mbar_try_wait(&bar, 0)) {
            if (++spins > kSpinLimit) {
                *ts.err = 2;
                break;
            }
        }
    }

    // ---- flags for ITEMS consecutive elements ----
    T x[ITEMS];
    {
        const uint4* row = reinterpret_cast<const uint4*>(buf + tid * ITEMS);
#pragma unroll
        for (int v = 0; v < kVpt; ++v) {
            uint4 r = row[v];
            const T* e = reinterpret_cast<const T*>(&r);
#pragma unroll
            for (int k = 0; k < V; ++k) x[v * V + k] = e[k];
        }
    }
    const uint32_t row0 = (uint32_t)tid * ITEMS;
    uint32_t flags = 0;
    if constexpr (MODE == 1) {
        T prev = tid > 0 ? buf[row0 - 1] : prev_of_tile;
        const bool first_global = (base == 0 && tid == 0);
#pragma unroll
        for (int j = 0; j < ITEMS; ++j) {
            const bool keep = (j == 0 && first_global) || !(x[j] == (j ? x[j - 1] : prev));
            if (row0 + j < cnt && keep) flags |= 1u << j;
        }
    } else {
#pragma unroll
        for (int j = 0; j < ITEMS; ++j)
            if (row0 + j < cnt && pred(x[j])) flags |= 1u << j;
    }

    // ---- ranks within the tile ----
    const uint32_t c = __popc(flags);
    const uint32_t incl = warp_inclusive_scan(c, OpSum());
    uint32_t texcl = shfl_up(incl, 1);
    if (lane == 0) texcl = 0;
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        const uint32_t w = lane < kBlock / 32 ? s_warp[lane] : 0u;
        const uint32_t wi = warp_inclusive_scan(w, OpSum());
        const uint32_t agg = shfl_idx(wi, kBlock / 32 - 1);
        uint32_t wex = shfl_up(wi, 1);
        if (lane == 0) wex = 0;
        const uint64_t prefix = lookback<uint64_t>(ts, tile, (uint64_t)agg);
        if (lane < kBlock / 32) s_wex[lane] = wex;
        if (lane == 0) {
            s_prefix = prefix;
            s_kept = agg;
            if (MODE != 2 && tile == gridDim.x - 1) *count_out = prefix + agg;
        }
    }
    __syncthreads();
    const uint32_t tile_kept = s_kept;
    const uint64_t prefix = s_prefix;
    uint32_t r = s_wex[warp] + texcl;  // tile-local rank of this thread's first kept element

    // ---- pack into shared memory (all rows were read before the barrier above) ----
    if constexpr (MODE == 2) {
        uint32_t rf = row0 - r;  // rejected elements before this thread's row, within the tile
#pragma unroll
        for (int j = 0; j < ITEMS; ++j) {
            if (row0 + j >= cnt) break;
            if (flags >> j & 1u) buf[r++] = x[j];
            else buf[tile_kept + rf++] = x[j];
        }
    } else {
#pragma unroll
        for (int j = 0; j < ITEMS; ++j)
            if (flags >> j & 1u) buf[r++] = x[j];
    }
    __syncthreads();

    // ---- coalesced stores ----
    if constexpr (MODE == 2) {
        const uint64_t nt = *num_true;
        const uint64_t rej_base = nt + (base - prefix);
        for (uint32_t i = tid; i < cnt; i += kBlock) {
            const uint64_t dst = i < tile_kept ? prefix + i : rej_base + (i - tile_kept);
            if (dst < n) out[dst] = buf[i];
            else *ts.err = 3;  // only reachable after a failed wait: never write out of range
        }
        if (tid == 0 && tile == gridDim.x - 1) *count_out = nt;
    } else {
        for (uint32_t i = tid; i < tile_kept; i += kBlock) {
            if (prefix + i < n) out[prefix + i] = buf[i];
            else *ts.err = 3;
        }
    }
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
    return e;
}

template <typename T, int MODE>
void launch_mode(dim3 grid, cudaStream_t s, bool bulk, const T* in, T* out, uint64_t n,
                 PredDev<T> p, TileStatus<uint64_t> ts, const unsigned long long* nt,
                 unsigned long long* count_out) {
    if (bulk) k_compact<T, MODE, true><<<grid, kBlock, 0, s>>>(in, out, n, p, ts, nt, count_out);
    else k_compact<T, MODE, false><<<grid, kBlock, 0, s>>>(in, out, n, p, ts, nt, count_out);
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
    if (mode == CompactMode::PARTITION) {
        // count pass: k = |{i : pred(in[i])}| into device scratch
        if (!launch_count_if(ws, dtype_of<T>(), pr, d_in, n, reinterpret_cast<uint64_t*>(nt)))
            return false;
    }
    auto ts = tile_status_at<uint64_t>(scratch, ws.next_epoch(), &ws.d_slot->spin_error);
    const bool bulk = reinterpret_cast<uintptr_t>(d_in) % 16 == 0;
    const T* in = static_cast<const T*>(d_in);
    T* out = static_cast<T*>(d_out);
    auto* cnt_out = reinterpret_cast<unsigned long long*>(d_count);
    PredDev<T> p = make_pred<T>(pr);
    dim3 grid((unsigned)tiles);
    cudaStream_t s = ws.stream();
    // profile bytes: input read (+ the kept elements written, known only on the device)
    ProfScope prof(ws, mode == CompactMode::PARTITION ? "k_partition"
                       : mode == CompactMode::UNIQUE ? "k_unique" : "k_copy_if",
                   (mode == CompactMode::PARTITION ? 2 : 1) * n * sizeof(T));
    switch (mode) {
        case CompactMode::SELECT:
            launch_mode<T, 0>(grid, s, bulk, in, out, n, p, ts, nt, cnt_out);
            break;
        case CompactMode::UNIQUE:
            launch_mode<T, 1>(grid, s, bulk, in, out, n, p, ts, nt, cnt_out);
            break;
        case CompactMode::PARTITION:
            launch_mode<T, 2>(grid, s, bulk, in, out, n, p, ts, nt, cnt_out);
            break;
    }
    count_launch();
    return cuda_ok(cudaGetLastError(), "k_compact launch");
}

}  // namespace

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
