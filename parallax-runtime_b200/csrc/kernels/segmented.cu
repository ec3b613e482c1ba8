// Segmented primitives: thousands of uneven segments in ONE persistent launch.
//
// No reference counterpart (the reference dispatches one primitive call per array,
// src/kernel/kernel_launcher.cpp); this is the batching path of the B200 design.
//
// Segments are either CSR (`offsets`, device, num_segments + 1 entries, cut one input
// array) or descriptors (one device-resident SegDesc per segment with its own addresses,
// used by the serving loop to coalesce requests without moving their operands). A one-CTA
// planner kernel turns the segment lengths into a tile work list (item_start[s] = first work
// item of segment s; a segment of L elements has ceil(L / TILE) items) and writes the
// results of empty segments; a second small kernel inverts it (item -> segment). The
// persistent kernel's CTAs then claim work items from an atomic counter in order, look up
// their segment, and process one tile each:
//   reduce   tile sum -> per-item partial; the last tile of a segment to finish (per-
//            segment ticket) folds the segment's partials in item order (deterministic)
//   scan     tile scan + decoupled look-back that stops at the segment's first tile
//            (exclusive with an init value, or inclusive)
//   copy_if  flags + tile ranks + look-back on kept counts within the segment; kept
//            elements of segment s land at the start of its output, its count in its slot
// TILE = 256 threads x ITEMS; ITEMS (4, 8 or 16) is picked per (primitive, element type,
// average segment length bucket) by timing the candidates on the first call (autotuner).
// Every CSR launch sequence (planner + persistent kernel) is captured once per argument
// set as a CUDA graph and replayed; the look-back epoch lives in device memory and is
// advanced by the planner, so a replay never reads status words of an earlier replay.
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

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

constexpr int kBlock = 256;
constexpr int kCandidates[3] = {4, 8, 16};

constexpr int SEG_REDUCE = (int)SegKind::REDUCE;
constexpr int SEG_SCAN = (int)SegKind::SCAN;
constexpr int SEG_COPY_IF = (int)SegKind::COPY_IF;

// Device buffers of one segmented launch (the workspace's segment and status buffers).
struct SegBuffers {
    uint32_t* item_start;  // num_segments + 1
    uint32_t* item_seg;    // one per work item: its segment (k_seg_map)
    uint32_t* tickets;     // num_segments, zeroed by the planner
    uint64_t* partials;    // one per work item
    StatusEntry* status;   // one per work item (a buffer of its own)
    uint64_t status_cap;   // entries in that buffer
    uint32_t* counters;    // [0] claim, [1] exit, [2] epoch, [3] error
};

// ---- tile loads ----------------------------------------------------------------------------------
// Loads `len` (<= 256 * ITEMS) elements starting at `src` into shared memory, striped (coalesced),
// padding with `pad`; afterwards thread t's row is sm[t*ITEMS, t*ITEMS + ITEMS).
template <typename T, int ITEMS>
__device__ __forceinline__ void load_tile(T* sm, const T* src, uint32_t len, T pad) {
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) {
        const uint32_t e = (uint32_t)k * kBlock + threadIdx.x;
        sm[e] = e < len ? src[e] : pad;
    }
}

template <typename T, typename A>
__device__ __forceinline__ A block_sum(A v, A* red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    v = warp_reduce(v, OpSum());
    if (lane == 0) red[warp] = v;
    __syncthreads();
    A t = A(0);
#pragma unroll
    for (int w = 0; w < kBlock / 32; ++w) t = t + red[w];
    __syncthreads();
    return t;
}

template <typename T>
struct SegPred {
    PredKind kind;
    bool negate;
    T c;
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
            default: v = false; break;
        }
        return v != negate;
    }
};

template <typename T> struct SegAcc { using type = typename SumAcc<T>::type; };

// ---- the persistent kernel -------------------------------------------------------------------------
template <typename T, int ITEMS, int OP>
__global__ void __launch_bounds__(kBlock)
k_segmented(SegSrc src, uint64_t S, SegBuffers b, T init, bool inclusive, SegPred<T> pred,
            volatile int32_t* err) {
    using A = typename SegAcc<T>::type;
    constexpr int TILE = kBlock * ITEMS;
    __shared__ __align__(16) T sm[TILE];
    __shared__ A red[kBlock / 32 + 1];
    __shared__ uint64_t red64[kBlock / 32 + 1];
    __shared__ int first[kBlock / 32];
    __shared__ uint32_t s_item;
    __shared__ uint32_t s_seg;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t total = b.item_start[S];
    TileStatus<A> ts;
    ts.e = b.status;
    ts.epoch = b.counters[2];
    ts.err = err;
    TileStatus<uint64_t> tsk;
    tsk.e = b.status;
    tsk.epoch = b.counters[2];
    tsk.err = err;

    for (;;) {
        if (tid == 0) {
            const uint32_t item = atomicAdd(&b.counters[0], 1u);
            s_item = item;
            s_seg = item < total ? b.item_seg[item] : 0u;
        }
        __syncthreads();
        const uint32_t item = s_item;
        const uint32_t seg = s_seg;
        __syncthreads();
        if (item >= total) break;
        const uint32_t first_item = b.item_start[seg];
        const uint32_t seg_items = b.item_start[seg + 1] - first_item;
        const uint32_t k = item - first_item;  // tile index within the segment
        const uint64_t seg_len = src.len(seg);
        const T* in = reinterpret_cast<const T*>(src.in_addr(seg));
        T* out = reinterpret_cast<T*>(src.out_addr(seg));
        const uint64_t begin = (uint64_t)k * TILE;  // within the segment
        const uint32_t len = (uint32_t)min((uint64_t)TILE, seg_len - begin);

        if constexpr (OP == SEG_REDUCE) {
            A acc = A(0);
#pragma unroll
            for (int j = 0; j < ITEMS; ++j) {
                const uint32_t e = (uint32_t)j * kBlock + tid;
                if (e < len) acc = acc + (A)in[begin + e];
            }
            const A sum = block_sum<T, A>(acc, red);
            T* res = reinterpret_cast<T*>(src.aux_addr(seg));
            if (seg_items == 1) {
                if (tid == 0) *res = (T)sum;
            } else {
                __shared__ bool s_last;
                if (tid == 0) {
                    put_val(&b.partials[item], sum);
                    __threadfence();
                    s_last = atomicAdd(&b.tickets[seg], 1u) == seg_items - 1;
                }
                __syncthreads();
                if (s_last) {  // fold the segment's partials in item order
                    __threadfence();
                    A f = A(0);
                    for (uint32_t i = tid; i < seg_items; i += kBlock)
                        f = f + get_val<A>(&b.partials[first_item + i]);
                    const A t = block_sum<T, A>(f, red);
                    if (tid == 0) *res = (T)t;
                }
                __syncthreads();
            }
        } else if constexpr (OP == SEG_SCAN) {
            load_tile<T, ITEMS>(sm, in + begin, len, T(0));
            __syncthreads();
            A x[ITEMS];
#pragma unroll
            for (int j = 0; j < ITEMS; ++j) x[j] = (A)sm[tid * ITEMS + j];
#pragma unroll
            for (int j = 1; j < ITEMS; ++j) x[j] = x[j - 1] + x[j];
            const A incl = warp_inclusive_scan(x[ITEMS - 1], OpSum());
            A tex = shfl_up(incl, 1);
            if (lane == 0) tex = A(0);
            if (lane == 31) red[warp] = incl;
            __syncthreads();
            A woff = A(0), agg = A(0);
#pragma unroll
            for (int w = 0; w < kBlock / 32; ++w) {
                if (w < warp) woff = woff + red[w];
                agg = agg + red[w];
            }
            __syncthreads();
            const A prefix = lookback_cta<A, kBlock>(ts, item, agg, red, first, first_item);
            const A tb = (A)init + ((prefix + woff) + tex);
            if (inclusive) {
#pragma unroll
                for (int j = 0; j < ITEMS; ++j) sm[tid * ITEMS + j] = (T)(tb + x[j]);
            } else {
#pragma unroll
                for (int j = 0; j < ITEMS; ++j) sm[tid * ITEMS + j] = (T)(j == 0 ? tb : tb + x[j - 1]);
            }
            __syncthreads();
#pragma unroll
            for (int j = 0; j < ITEMS; ++j) {
                const uint32_t e = (uint32_t)j * kBlock + tid;
                if (e < len) out[begin + e] = sm[e];
            }
            __syncthreads();
        } else {  // SEG_COPY_IF
            load_tile<T, ITEMS>(sm, in + begin, len, T(0));
            __syncthreads();
            T x[ITEMS];
            uint32_t f = 0;
#pragma unroll
            for (int j = 0; j < ITEMS; ++j) {
                x[j] = sm[tid * ITEMS + j];
                if ((uint32_t)(tid * ITEMS + j) < len && pred(x[j])) f |= 1u << j;
            }
            const uint32_t c = __popc(f);
            const uint32_t incl = warp_inclusive_scan(c, OpSum());
            uint32_t tex = shfl_up(incl, 1);
            if (lane == 0) tex = 0;
            __shared__ uint32_t wcnt[kBlock / 32];
            if (lane == 31) wcnt[warp] = incl;
            __syncthreads();
            uint32_t woff = 0, kept = 0;
#pragma unroll
            for (int w = 0; w < kBlock / 32; ++w) {
                if (w < warp) woff += wcnt[w];
                kept += wcnt[w];
            }
            const uint64_t prefix =
                lookback_cta<uint64_t, kBlock>(tsk, item, (uint64_t)kept, red64, first, first_item);
            uint32_t r = woff + tex;
#pragma unroll
            for (int j = 0; j < ITEMS; ++j)
                if (f >> j & 1u) sm[r++] = x[j];  // rows were read before the barriers above
            __syncthreads();
            for (uint32_t i = tid; i < kept; i += kBlock) {
                if (prefix + i < seg_len) out[prefix + i] = sm[i];
                else *err = 3;
            }
            if (tid == 0 && k == seg_items - 1)
                *reinterpret_cast<uint64_t*>(src.aux_addr(seg)) = prefix + kept;
            __syncthreads();
        }
    }
    if (tid == 0) persistent_exit(b.counters);
}

// ---- host side: buffers, tuner, graphs ------------------------------------------------------------
size_t up256(size_t v) { return (v + 255) / 256 * 256; }

// Carves the buffers for S segments and at most `items` work items out of the workspace's
// segment buffer (zeroed when it is (re)allocated).
bool seg_buffers(Workspace& ws, uint64_t S, uint64_t items, SegBuffers* out) {
    const size_t need = 256 + up256((S + 1) * 4) + up256(S * 4) + up256(items * 8) +
                        up256(items * 4);
    char* p = static_cast<char*>(ws.seg(need));
    out->status = static_cast<StatusEntry*>(ws.seg_status(items));
    if (!p || !out->status) return false;
    out->status_cap = ws.seg_status_cap;
    out->counters = reinterpret_cast<uint32_t*>(p);
    p += 256;
    out->item_start = reinterpret_cast<uint32_t*>(p);
    p += up256((S + 1) * 4);
    out->tickets = reinterpret_cast<uint32_t*>(p);
    p += up256(S * 4);
    out->partials = reinterpret_cast<uint64_t*>(p);
    p += up256(items * 8);
    out->item_seg = reinterpret_cast<uint32_t*>(p);
    return true;
}

struct SegCall {
    int op;            // SEG_REDUCE / SEG_SCAN / SEG_COPY_IF
    DType t;
    SegSrc src;
    uint64_t S;
    uint64_t count;    // CSR: elements of the input array; descriptors: sum of lengths
    uint64_t init_bits;
    bool inclusive;
    bool tune;         // may time the tile candidates (launches must be idempotent)
    Pred pred;
};

template <typename T, int ITEMS>
bool enqueue_typed(Workspace& ws, const SegCall& c, const SegBuffers& b) {
    constexpr int TILE = kBlock * ITEMS;
    cudaStream_t s = ws.stream();
    volatile int32_t* err = &ws.d_slot->spin_error;
    const uint64_t items_cap = c.S + c.count / TILE + 1;  // bound on the planner's items
    const SegEmpty empty = c.op == SEG_REDUCE ? SegEmpty::ZERO_RESULT
                         : c.op == SEG_COPY_IF ? SegEmpty::ZERO_COUNT : SegEmpty::NONE;
    k_seg_plan<kBlock><<<1, kBlock, 0, s>>>(c.src, c.S, c.count, (uint32_t)TILE, b.item_start,
                                            b.counters, empty,
                                            c.op == SEG_REDUCE ? b.tickets : nullptr, b.status,
                                            b.status_cap, err,
                                            items_cap <= kInlineItems ? b.item_seg : nullptr);
    if (items_cap > kInlineItems)
        k_seg_map<256><<<seg_map_grid(c.S), 256, 0, s>>>(b.item_start, c.S, b.item_seg);
    T init;
    memcpy(&init, &c.init_bits, sizeof(T));
    SegPred<T> pr;
    pr.kind = c.pred.kind;
    pr.negate = c.pred.negate;
    pr.c = std::is_floating_point<T>::value ? (T)c.pred.f
         : std::is_signed<T>::value ? (T)c.pred.i : (T)c.pred.u;
    // resident CTAs per SM of this instantiation (queried once), and no more CTAs than work
    // items: a small batch launches a small grid
    static int per_sm_of[3] = {0, 0, 0};
    int& per_sm = per_sm_of[c.op];
    if (per_sm == 0) {
        void* kfn = nullptr;
        switch (c.op) {
            case SEG_REDUCE: kfn = (void*)k_segmented<T, ITEMS, SEG_REDUCE>; break;
            case SEG_SCAN: kfn = (void*)k_segmented<T, ITEMS, SEG_SCAN>; break;
            default: kfn = (void*)k_segmented<T, ITEMS, SEG_COPY_IF>; break;
        }
        int v = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, kfn, kBlock, 0);
        per_sm = v < 1 ? 1 : v;
    }
    const uint64_t resident = (uint64_t)per_sm * device_info().sm_count;
    const unsigned grid = (unsigned)(items_cap < resident ? items_cap : resident);
    switch (c.op) {
        case SEG_REDUCE:
            k_segmented<T, ITEMS, SEG_REDUCE><<<grid, kBlock, 0, s>>>(c.src, c.S, b, init, false, pr, err);
            break;
        case SEG_SCAN:
            k_segmented<T, ITEMS, SEG_SCAN><<<grid, kBlock, 0, s>>>(c.src, c.S, b, init, c.inclusive, pr, err);
            break;
        default:
            k_segmented<T, ITEMS, SEG_COPY_IF><<<grid, kBlock, 0, s>>>(c.src, c.S, b, init, false, pr, err);
            break;
    }
    return cuda_ok(cudaGetLastError(), "segmented launch");
}

template <typename T>
bool enqueue_items(Workspace& ws, const SegCall& c, int items) {
    const uint64_t tile_min = (uint64_t)kBlock * kCandidates[0];
    SegBuffers b;
    if (!seg_buffers(ws, c.S, c.S + c.count / tile_min + 1, &b)) return false;
    switch (items) {
        case 4: return enqueue_typed<T, 4>(ws, c, b);
        case 8: return enqueue_typed<T, 8>(ws, c, b);
        default: return enqueue_typed<T, 16>(ws, c, b);
    }
}

bool enqueue(Workspace& ws, const SegCall& c, int items) {
    switch (c.t) {
        case DType::F32: return enqueue_items<float>(ws, c, items);
        case DType::F64: return enqueue_items<double>(ws, c, items);
        case DType::I32: return enqueue_items<int32_t>(ws, c, items);
        case DType::I64: return enqueue_items<int64_t>(ws, c, items);
        case DType::U32: return enqueue_items<uint32_t>(ws, c, items);
        case DType::U64: return enqueue_items<uint64_t>(ws, c, items);
        default: break;
    }
    set_error(PARALLAX_ERR_INVALID_ARGUMENT, "segmented: unsupported element type");
    return false;
}

// ---- autotuner -----------------------------------------------------------------------------------
// Choice per (op, dtype, log2 of the average segment length); timed on the first call with
// those parameters, optionally persisted in PARALLAX_TUNE_CACHE ("op dtype bucket items").
std::mutex g_tune_mu;
std::map<std::tuple<int, int, int>, int>* g_tune = nullptr;

void tune_load_locked() {
    if (g_tune) return;
    g_tune = new std::map<std::tuple<int, int, int>, int>();
    const char* path = getenv("PARALLAX_TUNE_CACHE");
    if (!path) return;
    FILE* f = fopen(path, "r");
    if (!f) return;
    int op, t, bucket, items;
    while (fscanf(f, "%d %d %d %d", &op, &t, &bucket, &items) == 4)
        (*g_tune)[std::make_tuple(op, t, bucket)] = items;
    fclose(f);
}

void tune_store_locked() {
    const char* path = getenv("PARALLAX_TUNE_CACHE");
    if (!path) return;
    FILE* f = fopen(path, "w");
    if (!f) return;
    for (auto& kv : *g_tune)
        fprintf(f, "%d %d %d %d\n", std::get<0>(kv.first), std::get<1>(kv.first),
                std::get<2>(kv.first), kv.second);
    fclose(f);
}

int bucket_of(const SegCall& c) {
    uint64_t avg = c.S ? c.count / c.S : 0;
    int b = 0;
    while ((1ull << (b + 1)) <= avg && b < 30) ++b;
    return b;
}

// Returns the tile choice, timing the candidates (and leaving valid results) when unknown.
int tuned_items(Workspace& ws, const SegCall& c) {
    const auto key = std::make_tuple((int)c.op, (int)c.t, bucket_of(c));
    {
        std::lock_guard<std::mutex> g(g_tune_mu);
        tune_load_locked();
        auto it = g_tune->find(key);
        if (it != g_tune->end()) return it->second;
    }
    if (!c.tune || (getenv("PARALLAX_TUNE") && atoi(getenv("PARALLAX_TUNE")) == 0)) {
        const uint64_t avg = c.S ? c.count / c.S : 0;  // untuned: by average segment length
        return avg >= (16u << 10) ? 16 : avg >= (2u << 10) ? 8 : 4;
    }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    int best = 8;
    float best_ms = 1e30f;
    cudaStream_t s = ws.stream();
    for (int cand : kCandidates) {
        if (!enqueue(ws, c, cand)) break;  // warm-up (first-touch, module load)
        cudaEventRecord(e0, s);
        if (!enqueue(ws, c, cand)) break;
        cudaEventRecord(e1, s);
        if (cudaEventSynchronize(e1) != cudaSuccess) break;
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
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
        fprintf(stderr, "[parallax] tuned segmented op %d dtype %d bucket %d -> %d items/thread (%.3f ms)\n",
                (int)c.op, (int)c.t, bucket_of(c), best, best_ms);
    return best;
}

// ---- graph capture and replay -----------------------------------------------------------------
std::string graph_key(const SegCall& c, int items) {
    char k[512];
    snprintf(k, sizeof k, "%d/%d/%llx/%llx/%p/%llx/%llu/%llu/%llx/%d/%d/%d/%g/%lld/%llu/%d", c.op,
             (int)c.t, (unsigned long long)c.src.in, (unsigned long long)c.src.out,
             (const void*)c.src.offsets, (unsigned long long)c.src.aux, (unsigned long long)c.S,
             (unsigned long long)c.count, (unsigned long long)c.init_bits, (int)c.inclusive,
             (int)c.pred.kind, (int)c.pred.negate, c.pred.f, (long long)c.pred.i,
             (unsigned long long)c.pred.u, items);
    return k;
}

const char* op_name(int op) {
    return op == SEG_REDUCE ? "segmented_reduce"
         : op == SEG_SCAN ? "segmented_scan" : "segmented_copy_if";
}

// Sizes the buffers for the smallest tile before any capture (growth would invalidate a
// captured graph).
bool reserve(Workspace& ws, const SegCall& c) {
    const uint64_t tile_min = (uint64_t)kBlock * kCandidates[0];
    SegBuffers b;
    return seg_buffers(ws, c.S, c.S + c.count / tile_min + 1, &b);
}

bool run(Workspace& ws, const SegCall& c, bool graph) {
    const int items = tuned_items(ws, c);
    if (!reserve(ws, c)) return false;
    const size_t es = dtype_size(c.t);
    ProfScope prof(ws, op_name(c.op), (c.op == SEG_SCAN ? 2 : 1) * c.count * es);
    count_launch(3);
    if (!graph) return enqueue(ws, c, items);
    return graph_launch(ws, graph_key(c, items), [&] { return enqueue(ws, c, items); });
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
    void* d_aux = nullptr;  // results (reduce) or counts (copy_if); scans have none
    if (c.op != SEG_SCAN &&
        !(d_aux = device_operand(aux, fn, c.op == SEG_REDUCE ? "results" : "counts")))
        return last_error();
    if (c.S >= 0xffffffffull || c.count / ((uint64_t)kBlock * kCandidates[0]) + c.S >= 0xffffffffull) {
        set_error(PARALLAX_ERR_INVALID_ARGUMENT, "%s: too many segments / elements", fn);
        return PARALLAX_ERR_INVALID_ARGUMENT;
    }
    const uint32_t es = (uint32_t)dtype_size(c.t);
    c.src = SegSrc{static_cast<const uint64_t*>(d_off), nullptr, (uint64_t)d_in, (uint64_t)d_out,
                   (uint64_t)d_aux, c.op == SEG_COPY_IF ? 8u : es, es};
    if (!run(*ws, c, true)) return last_error() ? last_error() : PARALLAX_ERR_CUDA;
    return ws->async ? PARALLAX_OK : sync_stream(*ws);
}

}  // namespace

bool launch_segmented_descs(Workspace& ws, SegKind op, DType t, const Pred& p, bool inclusive,
                            uint64_t init_bits, const SegDesc* d_descs, uint64_t S,
                            uint64_t total) {
    if (S == 0) return true;
    if (S >= 0xffffffffull || total / ((uint64_t)kBlock * kCandidates[0]) + S >= 0xffffffffull) {
        set_error(PARALLAX_ERR_INVALID_ARGUMENT, "batched launch: too many segments / elements");
        return false;
    }
    SegCall c{};
    c.op = (int)op;
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
    Handle* h = as_handle(kernel);
    if (!h || h->kind != Kind::REDUCE || h->op != RedOp::SUM) {
        set_error(PARALLAX_ERR_INVALID_HANDLE, "parallax_segmented_reduce: needs a reduce:sum handle");
        return PARALLAX_ERR_INVALID_HANDLE;
    }
    SegCall c{};
    c.op = SEG_REDUCE;
    c.t = h->dtype;
    c.count = count;
    c.S = num_segments;
    c.tune = true;
    return seg_entry(c, data, nullptr, offsets, results, "parallax_segmented_reduce");
}

PXB_EXPORT int parallax_segmented_exclusive_scan(parallax_kernel_t kernel, const void* input,
                                                 void* output, size_t count,
                                                 const uint64_t* offsets, size_t num_segments,
                                                 const void* init) {
    Handle* h = as_handle(kernel);
    if (!h || h->kind != Kind::SCAN) {
        set_error(PARALLAX_ERR_INVALID_HANDLE, "parallax_segmented_exclusive_scan: needs a scan handle");
        return PARALLAX_ERR_INVALID_HANDLE;
    }
    SegCall c{};
    c.op = SEG_SCAN;
    c.t = h->dtype;
    c.count = count;
    c.S = num_segments;
    c.tune = input != output;  // timing the candidates in place would scan twice
    if (init) memcpy(&c.init_bits, init, dtype_size(h->dtype));
    return seg_entry(c, input, output, offsets, nullptr, "parallax_segmented_exclusive_scan");
}

PXB_EXPORT int parallax_segmented_copy_if(parallax_kernel_t kernel, const void* input,
                                          void* output, size_t count, const uint64_t* offsets,
                                          size_t num_segments, uint64_t* counts) {
    Handle* h = as_handle(kernel);
    if (!h || h->kind != Kind::COMPACT_FLAGS || h->pred.kind == PredKind::MOD) {
        set_error(PARALLAX_ERR_INVALID_HANDLE,
                  "parallax_segmented_copy_if: needs a copy_if / remove_if handle (comparison predicate)");
        return PARALLAX_ERR_INVALID_HANDLE;
    }
    SegCall c{};
    c.op = SEG_COPY_IF;
    c.t = h->dtype;
    c.count = count;
    c.S = num_segments;
    c.tune = true;
    c.pred = h->pred;
    if (h->remove) c.pred.negate = !c.pred.negate;
    return seg_entry(c, input, output, offsets, counts, "parallax_segmented_copy_if");
}
