// Ascending sort: bitonic tile sort in registers / shuffles / shared memory, then
// merge-path merge passes over HBM.
//
// Reference: a global bitonic network, one dispatch + fence wait per (k, j) stage,
// log2(n)(log2(n)+1)/2 passes over the whole array (351 at n = 2^26), n a power of two
// (src/kernel/kernel_launcher.cpp:1568-1606, shaders/bitonic.comp:15-29).
//
// Here the same compare-exchange network runs only inside 16 KiB tiles (4096 4-byte or
// 2048 8-byte keys per 256-thread CTA): stages whose partner distance j is below the
// per-thread run use registers, j up to 32 runs uses warp shuffles, larger j goes through
// shared memory. Sorted tiles are then merged pairwise, doubling the run length each
// pass: a CTA finds its output tiles' spans on the merge path (one warp per split, 32-ary
// search over HBM), stages the two input spans in shared memory and merges stably, each
// thread producing its 16 (8) contiguous outputs in registers. Any n is accepted (the
// last tile is padded with the largest key in registers only).
// Keys are sorted as unsigned integers after an order-preserving transform: signed
// integers flip the sign bit; IEEE floats flip all bits when negative and the sign bit
// otherwise (the IEEE total order: -0.0 sorts before +0.0). The transform is fused into
// the first load and its inverse into the last store. 8-byte records of the key-value
// sort are (key << 32 | value) and sort as plain 64-bit keys, i.e. stably by key.
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../runtime.hpp"
#include "../segplan.cuh"
#include "../sortkey.cuh"

namespace pxb {
namespace {

constexpr int kBlock = 256;

template <typename K> struct SortShape;
template <> struct SortShape<uint32_t> { static constexpr int ITEMS = 16; };
template <> struct SortShape<uint64_t> { static constexpr int ITEMS = 8; };

template <typename K>
__device__ __forceinline__ K kmin(K a, K b) { return b < a ? b : a; }
template <typename K>
__device__ __forceinline__ K kmax(K a, K b) { return b < a ? a : b; }

// ---- bitonic network, unrolled at compile time -------------------------------------------
// Thread t holds keys [t*ITEMS, t*ITEMS + ITEMS) of the tile in x[]. Stage (k, j) pairs
// element i with i ^ j, ascending when (i & k) == 0.
template <typename K, int ITEMS, int k, int j>
__device__ __forceinline__ void bitonic_stage(K (&x)[ITEMS], K* sm, int t, int lane, int row0) {
    if constexpr (j < ITEMS) {  // partner in the same thread
#pragma unroll
        for (int r = 0; r < ITEMS; ++r) {
            if (r & j) continue;
            const int r2 = r | j;
            const bool asc = (k < ITEMS) ? ((r & k) == 0) : ((row0 & k) == 0);
            const K a = x[r], b = x[r2];
            const K lo = kmin(a, b), hi = kmax(a, b);
            x[r] = asc ? lo : hi;
            x[r2] = asc ? hi : lo;
        }
    } else if constexpr (j < 32 * ITEMS) {  // partner in the same warp
        constexpr int m = j / ITEMS;
        const bool keep_min = ((lane & m) == 0) == ((row0 & k) == 0);
#pragma unroll
        for (int r = 0; r < ITEMS; ++r) {
            const K o = __shfl_xor_sync(0xffffffffu, x[r], m);
            x[r] = keep_min ? kmin(x[r], o) : kmax(x[r], o);
        }
    } else {  // partner in another warp: exchange through shared memory
        constexpr int m = j / ITEMS;
        const bool keep_min = ((t & m) == 0) == ((row0 & k) == 0);
        __syncthreads();
#pragma unroll
        for (int r = 0; r < ITEMS; ++r) sm[r * kBlock + t] = x[r];
        __syncthreads();
#pragma unroll
        for (int r = 0; r < ITEMS; ++r) {
            const K o = sm[r * kBlock + (t ^ m)];
            x[r] = keep_min ? kmin(x[r], o) : kmax(x[r], o);
        }
    }
}
template <typename K, int ITEMS, int k, int j>
__device__ __forceinline__ void bitonic_j(K (&x)[ITEMS], K* sm, int t, int lane, int row0) {
    bitonic_stage<K, ITEMS, k, j>(x, sm, t, lane, row0);
    if constexpr (j > 1) bitonic_j<K, ITEMS, k, j / 2>(x, sm, t, lane, row0);
}
template <typename K, int ITEMS, int TILE, int k>
__device__ __forceinline__ void bitonic_k(K (&x)[ITEMS], K* sm, int t, int lane, int row0) {
    bitonic_j<K, ITEMS, k, k / 2>(x, sm, t, lane, row0);
    if constexpr (k < TILE) bitonic_k<K, ITEMS, TILE, k * 2>(x, sm, t, lane, row0);
}

// ---- tile sort ----------------------------------------------------------------------------
template <typename K, int XF>
__global__ void __launch_bounds__(kBlock)
k_tile_sort(const K* in, K* out, uint64_t n, bool apply_inverse) {
    constexpr int ITEMS = SortShape<K>::ITEMS;
    constexpr int TILE = kBlock * ITEMS;
    constexpr int V = 16 / sizeof(K);
    __shared__ K sm[TILE];
    const int t = threadIdx.x, lane = t & 31;
    const uint64_t base = (uint64_t)blockIdx.x * TILE;
    const uint64_t rem = n - base;
    const int cnt = rem < (uint64_t)TILE ? (int)rem : TILE;
    const int row0 = t * ITEMS;

    K x[ITEMS];
    const bool full = cnt == TILE && (reinterpret_cast<uintptr_t>(in) % 16 == 0);
    if (full) {
        const uint4* src = reinterpret_cast<const uint4*>(in + base + row0);
#pragma unroll
        for (int v = 0; v < ITEMS / V; ++v) {
            uint4 r = src[v];
            const K* e = reinterpret_cast<const K*>(&r);
#pragma unroll
            for (int k = 0; k < V; ++k) x[v * V + k] = to_key<K, XF>(e[k]);
        }
    } else {
#pragma unroll
        for (int r = 0; r < ITEMS; ++r)
            x[r] = row0 + r < cnt ? to_key<K, XF>(in[base + row0 + r]) : ~K(0);
    }

    bitonic_k<K, ITEMS, TILE, 2>(x, sm, t, lane, row0);

    if (full && (reinterpret_cast<uintptr_t>(out) % 16 == 0)) {
        uint4* dst = reinterpret_cast<uint4*>(out + base + row0);
#pragma unroll
        for (int v = 0; v < ITEMS / V; ++v) {
            uint4 r;
            K* e = reinterpret_cast<K*>(&r);
#pragma unroll
            for (int k = 0; k < V; ++k)
                e[k] = apply_inverse ? from_key<K, XF>(x[v * V + k]) : x[v * V + k];
            dst[v] = r;
        }
    } else {
#pragma unroll
        for (int r = 0; r < ITEMS; ++r)
            if (row0 + r < cnt)
                out[base + row0 + r] = apply_inverse ? from_key<K, XF>(x[r]) : x[r];
    }
}

// ---- merge path ---------------------------------------------------------------------------
// Pair geometry of output tile `o`: runs A = [ps, ps+la) and B = [ps+la, ps+la+lb).
// L (the run length) is a power of two.
struct Pair {
    uint64_t ps, la, lb;
};
__device__ __forceinline__ Pair pair_of(uint64_t o, uint64_t n, uint64_t L) {
    Pair p;
    p.ps = o & ~(2 * L - 1);
    const uint64_t r = n - p.ps;
    p.la = r < L ? r : L;
    const uint64_t r2 = r - p.la;
    p.lb = r2 < L ? r2 : L;
    return p;
}

// Warp-collective merge-path search: the number of A elements among the first d outputs
// of the stable merge of A[0, la) and B[0, lb) (A wins ties): the number of i < d with
// B[d-1-i] >= A[i] (a monotone predicate), found by a 32-ary search (32 probes a round).
template <typename K>
__device__ __forceinline__ uint64_t warp_merge_split(const K* __restrict__ A, uint64_t la,
                                                     const K* __restrict__ B, uint64_t lb,
                                                     uint64_t d) {
    const int lane = threadIdx.x & 31;
    uint64_t lo = d > lb ? d - lb : 0;
    uint64_t hi = d < la ? d : la;
    while (hi - lo > 32) {
        const uint64_t stride = (hi - lo + 31) / 32;
        const uint64_t q = lo + (uint64_t)lane * stride;
        const bool valid = q < hi;
        const bool tr = valid && !(B[d - 1 - q] < A[q]);
        const int c = __popc(__ballot_sync(0xffffffffu, tr));
        const int nvalid = __popc(__ballot_sync(0xffffffffu, valid));
        const uint64_t nlo = c ? lo + (uint64_t)(c - 1) * stride + 1 : lo;
        const uint64_t nhi = c < nvalid ? lo + (uint64_t)c * stride : hi;
        lo = nlo;
        hi = nhi;
    }
    const uint64_t q = lo + lane;
    const bool tr = q < hi && !(B[d - 1 - q] < A[q]);
    return lo + __popc(__ballot_sync(0xffffffffu, tr));
}

// The spans of one output tile: [a_s, a_e) of run A and [b_s, b_e) of run B, at most ot
// elements together. Sorted runs always give consistent spans; anything else is refused
// before a single element is staged.
__device__ __forceinline__ bool spans_ok(uint64_t a_s, uint64_t a_e, uint64_t b_s, uint64_t b_e,
                                         int ot) {
    return a_s <= a_e && b_s <= b_e && (a_e - a_s) + (b_e - b_s) <= (uint64_t)ot;
}

// Staged layout of a tile's two spans in shared memory: each span keeps the position of
// its first element within a 16-byte word (its phase), so it is staged with aligned
// 16-byte vector loads and stores: A[i] at sm[pa + i] (pa = A's phase), IPT sentinel keys
// (all ones, the largest transformed key) after it, B[j] at sm[bb + pb + j] (bb a
// 16-byte-aligned start after A's sentinels), IPT sentinels after B. A thread whose run in
// one span is exhausted keeps reading sentinels, which never win against a real key (a real
// key equal to the sentinel has the same bits, so either choice writes the same output),
// so the merge loop needs no bounds checks. The vectors at a span's two ends may carry up
// to 16 - sizeof(K) bytes from outside the span; an aligned 16-byte word that holds one
// byte of the span lies in the same memory page, so those reads cannot fault, and the
// extra elements land in slots that the sentinels overwrite or nothing reads.
template <typename K>
constexpr int staged_elems(int ot) { return ot + 2 * SortShape<K>::ITEMS + 4 * (16 / (int)sizeof(K)); }

// Merges the sorted spans As[0, na) and Bs[0, nb) (shared memory, sentinels after each,
// na + nb <= OT, A wins ties) into dst[0, na + nb): every thread finds its start on the
// merge path by binary search and merges its IPT outputs in registers (one shared load per
// output), then stores them as 16-byte vectors (a thread's outputs are contiguous).
template <typename K, int XF>
__device__ __forceinline__ void merge_spans(const K* As, int na, const K* Bs, int nb,
                                            K* __restrict__ dst, bool final_pass) {
    constexpr int IPT = SortShape<K>::ITEMS;
    constexpr int V = 16 / sizeof(K);
    const int total = na + nb;
    const int dt = threadIdx.x * IPT < total ? threadIdx.x * IPT : total;
    int lo = dt > nb ? dt - nb : 0, hi = dt < na ? dt : na;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (!(Bs[dt - 1 - mid] < As[mid])) lo = mid + 1;
        else hi = mid;
    }
    const K* pa = As + lo;
    const K* pb = Bs + (dt - lo);
    K a = *pa;
    K b = *pb;
    K out[IPT];
#pragma unroll
    for (int k = 0; k < IPT; ++k) {
        const bool take_a = !(b < a);
        out[k] = take_a ? a : b;
        pa += take_a;
        pb += !take_a;
        const K x = *(take_a ? pa : pb);
        a = take_a ? x : a;
        b = take_a ? b : x;
    }
    if (final_pass) {
#pragma unroll
        for (int k = 0; k < IPT; ++k) out[k] = from_key<K, XF>(out[k]);
    }
    if (dt + IPT <= total && (reinterpret_cast<uintptr_t>(dst) % 16 == 0)) {
        uint4* d = reinterpret_cast<uint4*>(dst + dt);
#pragma unroll
        for (int v = 0; v < IPT / V; ++v) {
            uint4 r;
            memcpy(&r, &out[v * V], 16);
            d[v] = r;
        }
    } else {
#pragma unroll
        for (int k = 0; k < IPT; ++k)
            if (dt + k < total) dst[dt + k] = out[k];
    }
}

// Where a tile's two spans sit in the staged layout above.
struct SpanPlace {
    int pa, pb;    // phases (element offset within a 16-byte word)
    int nva, nvb;  // 16-byte vectors per span
    int bb;        // B's vector-aligned start
};
template <typename K>
__device__ __forceinline__ SpanPlace span_place(const K* A, int na, const K* B, int nb) {
    constexpr int IPT = SortShape<K>::ITEMS;
    constexpr int V = 16 / sizeof(K);
    SpanPlace q;
    q.pa = (int)((reinterpret_cast<uintptr_t>(A) / sizeof(K)) % V);
    q.pb = (int)((reinterpret_cast<uintptr_t>(B) / sizeof(K)) % V);
    q.nva = na ? (q.pa + na + V - 1) / V : 0;
    q.nvb = nb ? (q.pb + nb + V - 1) / V : 0;
    q.bb = (q.pa + na + IPT + V - 1) / V * V;
    return q;
}
template <typename K>
constexpr int stage_vectors() {  // vectors per thread over both spans
    return (kBlock * SortShape<K>::ITEMS + 2 * (16 / (int)sizeof(K))) / (16 / (int)sizeof(K)) /
               kBlock + 1;
}
// Issues a thread's aligned 16-byte loads of both spans into registers.
template <typename K>
__device__ __forceinline__ void stage_load(const K* A, const K* B, const SpanPlace& q,
                                           uint4 (&r)[stage_vectors<K>()]) {
    const uint4* Av = reinterpret_cast<const uint4*>(A - q.pa);
    const uint4* Bv = reinterpret_cast<const uint4*>(B - q.pb);
#pragma unroll
    for (int k = 0; k < stage_vectors<K>(); ++k) {
        const int v = threadIdx.x + k * kBlock;
        if (v < q.nva) r[k] = Av[v];
        else if (v < q.nva + q.nvb) r[k] = Bv[v - q.nva];
    }
}
// Stores the registers into the staged layout and adds the sentinels (two barriers).
template <typename K>
__device__ __forceinline__ void stage_store(K* sm, int na, int nb, const SpanPlace& q,
                                            const uint4 (&r)[stage_vectors<K>()]) {
    constexpr int IPT = SortShape<K>::ITEMS;
    const int t = threadIdx.x;
#pragma unroll
    for (int k = 0; k < stage_vectors<K>(); ++k) {
        const int v = t + k * kBlock;
        if (v < q.nva) reinterpret_cast<uint4*>(sm)[v] = r[k];
        else if (v < q.nva + q.nvb) reinterpret_cast<uint4*>(sm + q.bb)[v - q.nva] = r[k];
    }
    __syncthreads();  // the vectors' extra elements are in place before the sentinels
    if (t < IPT) sm[q.pa + na + t] = ~K(0);
    else if (t < 2 * IPT) sm[q.bb + q.pb + nb + t - IPT] = ~K(0);
    __syncthreads();
}

// Stages A[0, na) and B[0, nb) in sm (staged_elems(OT) elements, the layout above) with
// aligned 16-byte loads, all of a thread's vectors of both spans in flight at once, then
// merges them.
template <typename K, int XF>
__device__ __forceinline__ void merge_tile(const K* __restrict__ A, int na, const K* __restrict__ B,
                                           int nb, K* __restrict__ dst, bool final_pass, K* sm) {
    const SpanPlace q = span_place(A, na, B, nb);
    uint4 r[stage_vectors<K>()];
    stage_load(A, B, q, r);
    stage_store(sm, na, nb, q, r);
    merge_spans<K, XF>(sm + q.pa, na, sm + q.bb + q.pb, nb, dst, final_pass);
}

// One CTA per `tpc` (1..kTilesPerCta) output tiles of OT keys. Each of the first 2 x tpc
// warps finds one tile start or end on the merge path of the tile's run pair (a 32-ary
// search over HBM, all searches in parallel, so the latency is paid once per CTA); the CTA
// then stages and merges its tiles in turn. Sorts of 2048 tiles or more use four tiles per
// CTA; smaller ones use one, for more CTAs and shorter ones.
constexpr int kTilesPerCta = 4;
static_assert(2 * kTilesPerCta <= kBlock / 32, "one warp per split");

template <typename K, int XF, bool FINAL, int TPC>
__global__ void __launch_bounds__(kBlock)
k_merge(const K* __restrict__ src, K* __restrict__ dst, uint64_t n, uint64_t L, uint64_t tiles,
        volatile int32_t* err) {
    constexpr int tpc = TPC;
    constexpr int OT = kBlock * SortShape<K>::ITEMS;
    __shared__ __align__(16) K sm[staged_elems<K>(OT)];
    __shared__ uint64_t s_split[2 * TPC];
    const uint64_t tile0 = (uint64_t)blockIdx.x * tpc;
    const int ntiles = (int)(tiles - tile0 < (uint64_t)tpc ? tiles - tile0 : tpc);
    const int warp = threadIdx.x >> 5;
    if (warp < 2 * ntiles) {
        const uint64_t o = (tile0 + warp / 2) * OT;
        const Pair p = pair_of(o, n, L);
        const uint64_t pair_end = p.ps + p.la + p.lb;
        const uint64_t d = (warp & 1) ? (o + OT < pair_end ? o + OT : pair_end) - p.ps : o - p.ps;
        const uint64_t v = ((warp & 1) && d == p.la + p.lb) ? p.la
                         : warp_merge_split(src + p.ps, p.la, src + p.ps + p.la, p.lb, d);
        if ((threadIdx.x & 31) == 0) s_split[warp] = v;
    }
    __syncthreads();
    struct Span {
        const K* a;
        const K* b;
        int na, nb;
        bool ok;
    };
    auto span = [&](int k) {
        const uint64_t o = (tile0 + k) * OT;
        const Pair p = pair_of(o, n, L);
        const uint64_t pair_end = p.ps + p.la + p.lb;
        const uint64_t d0 = o - p.ps, d1 = (o + OT < pair_end ? o + OT : pair_end) - p.ps;
        const uint64_t a_s = s_split[2 * k], a_e = s_split[2 * k + 1];
        const uint64_t b_s = d0 - a_s, b_e = d1 - a_e;
        Span sp;
        sp.ok = spans_ok(a_s, a_e, b_s, b_e, OT);  // else refused, never staged
        sp.a = src + p.ps + a_s;
        sp.b = src + p.ps + p.la + b_s;
        sp.na = sp.ok ? (int)(a_e - a_s) : 0;
        sp.nb = sp.ok ? (int)(b_e - b_s) : 0;
        return sp;
    };
    // The next tile's vectors are loaded into registers while the current tile merges.
    uint4 r[stage_vectors<K>()];
    Span cur = span(0);
    SpanPlace q = span_place(cur.a, cur.na, cur.b, cur.nb);
    stage_load(cur.a, cur.b, q, r);
    for (int k = 0; k < ntiles; ++k) {
        if (k) __syncthreads();  // the previous tile's shared-memory reads are done
        if (!cur.ok && threadIdx.x == 0) *err = kErrMergeSpan;
        stage_store(sm, cur.na, cur.nb, q, r);
        const K* As = sm + q.pa;
        const K* Bs = sm + q.bb + q.pb;
        const int na = cur.na, nb = cur.nb;
        if (k + 1 < ntiles) {
            cur = span(k + 1);
            q = span_place(cur.a, cur.na, cur.b, cur.nb);
            stage_load(cur.a, cur.b, q, r);
        }
        merge_spans<K, XF>(As, na, Bs, nb, dst + (tile0 + k) * OT, FINAL);
    }
}

template <typename K, int XF>
bool sort_keys(Workspace& ws, void* d_data, uint64_t n) {
    constexpr int TILE = kBlock * SortShape<K>::ITEMS;
    const uint64_t tiles = (n + TILE - 1) / TILE;
    if (tiles > 0x7fffffffull) {
        set_error(PARALLAX_ERR_INVALID_ARGUMENT, "sort: too many elements");
        return false;
    }
    int passes = 0;
    while ((uint64_t(1) << passes) < tiles) ++passes;
    K* data = static_cast<K*>(d_data);
    K* tmp = nullptr;
    if (passes) {
        tmp = static_cast<K*>(ws.temp(n * sizeof(K)));
        if (!tmp) return false;
    }
    cudaStream_t s = ws.stream();
    K* cur = (passes % 2 == 0) ? data : tmp;
    {
        ProfScope prof(ws, "k_tile_sort", 2 * n * sizeof(K));
        k_tile_sort<K, XF><<<(unsigned)tiles, kBlock, 0, s>>>(data, cur, n, passes == 0);
    }
    count_launch();
    for (int pass = 1; pass <= passes; ++pass) {
        const uint64_t L = (uint64_t)TILE << (pass - 1);
        K* nxt = cur == data ? tmp : data;
        {
            ProfScope prof(ws, "k_merge", 2 * n * sizeof(K));
            // four tiles per CTA from 2048 tiles (512 CTAs) up, one below
            volatile int32_t* err = &ws.d_slot->spin_error;
            if (tiles >= 2048) {
                const unsigned grid = (unsigned)((tiles + kTilesPerCta - 1) / kTilesPerCta);
                if (pass == passes)
                    k_merge<K, XF, true, kTilesPerCta><<<grid, kBlock, 0, s>>>(cur, nxt, n, L, tiles, err);
                else
                    k_merge<K, XF, false, kTilesPerCta><<<grid, kBlock, 0, s>>>(cur, nxt, n, L, tiles, err);
            } else {
                if (pass == passes)
                    k_merge<K, XF, true, 1><<<(unsigned)tiles, kBlock, 0, s>>>(cur, nxt, n, L, tiles, err);
                else
                    k_merge<K, XF, false, 1><<<(unsigned)tiles, kBlock, 0, s>>>(cur, nxt, n, L, tiles, err);
            }
        }
        count_launch(1);
        cur = nxt;
    }
    return cuda_ok(cudaGetLastError(), "sort launch");
}

// ---- segmented sort ---------------------------------------------------------------------------
// Work list from the planner with one item per TILE keys of a segment. A segment of m items
// needs P = ceil(log2 m) merge passes; its tile sort writes to the segment's data when P is
// even and to its temporary when P is odd, and every pass flips the buffer, so each segment
// ends in its data after its own last pass with no extra copy. Passes beyond a segment's P
// skip it. Segments are CSR (one array, temporary at the same offsets of one buffer) or
// descriptors (each with its own data and temporary addresses).
__device__ __forceinline__ int passes_of(uint32_t m) {
    int p = 0;
    while ((1u << p) < m) ++p;
    return p;
}

template <typename K>
struct SegGeom {
    uint32_t seg, first, m, k;
    uint64_t len;
    K* data;
    K* tmp;
    int P;
    // buffer holding the segment after q merge passes
    __device__ __forceinline__ K* loc(int q) const { return ((P - q) & 1) ? tmp : data; }
};
template <typename K>
__device__ __forceinline__ SegGeom<K> seg_geom(const SegSrc& src, const uint32_t* item_start,
                                               const uint32_t* item_seg, uint32_t item) {
    SegGeom<K> g;
    g.seg = item_seg[item];
    g.first = item_start[g.seg];
    g.m = item_start[g.seg + 1] - g.first;
    g.k = item - g.first;
    g.len = src.len(g.seg);
    g.data = reinterpret_cast<K*>(src.in_addr(g.seg));
    g.tmp = reinterpret_cast<K*>(src.aux_addr(g.seg));
    g.P = passes_of(g.m);
    return g;
}

template <typename K, int XF>
__global__ void __launch_bounds__(kBlock)
k_seg_tile_sort(SegSrc src, uint64_t S, const uint32_t* __restrict__ item_start,
                const uint32_t* __restrict__ item_seg) {
    constexpr int ITEMS = SortShape<K>::ITEMS;
    constexpr int TILE = kBlock * ITEMS;
    __shared__ K sm[TILE];
    const uint32_t item = blockIdx.x;
    if (item >= item_start[S]) return;
    const SegGeom<K> g = seg_geom<K>(src, item_start, item_seg, item);
    const int t = threadIdx.x, lane = t & 31, row0 = t * ITEMS;
    const uint64_t begin = (uint64_t)g.k * TILE;
    const uint64_t rem = g.len - begin;
    const int cnt = rem < (uint64_t)TILE ? (int)rem : TILE;
    const K* in = g.data + begin;
    K x[ITEMS];
#pragma unroll
    for (int r = 0; r < ITEMS; ++r) x[r] = row0 + r < cnt ? to_key<K, XF>(in[row0 + r]) : ~K(0);
    bitonic_k<K, ITEMS, TILE, 2>(x, sm, t, lane, row0);
    K* dst = g.loc(0) + begin;
#pragma unroll
    for (int r = 0; r < ITEMS; ++r)
        if (row0 + r < cnt) dst[row0 + r] = g.P == 0 ? from_key<K, XF>(x[r]) : x[r];
}

// One CTA per work item (output tile of OT keys) of every segment still merging in this
// pass; like k_merge, warps 0 and 1 find the tile's span on the merge path first.
template <typename K, int XF>
__global__ void __launch_bounds__(kBlock)
k_seg_merge(SegSrc src, uint64_t S, const uint32_t* __restrict__ item_start,
            const uint32_t* __restrict__ item_seg, int pass, volatile int32_t* err) {
    constexpr int OT = kBlock * SortShape<K>::ITEMS;
    __shared__ __align__(16) K sm[staged_elems<K>(OT)];
    __shared__ uint64_t s_split[2];
    const uint32_t item = blockIdx.x;
    if (item >= item_start[S]) return;
    const SegGeom<K> g = seg_geom<K>(src, item_start, item_seg, item);
    if (g.P < pass) return;
    const K* srcb = g.loc(pass - 1);
    const uint64_t L = (uint64_t)OT << (pass - 1);
    const uint64_t o = (uint64_t)g.k * OT;
    const Pair p = pair_of(o, g.len, L);
    const uint64_t pair_end = p.ps + p.la + p.lb;
    const uint64_t tile_end = o + OT < pair_end ? o + OT : pair_end;
    const uint64_t d0 = o - p.ps, d1 = tile_end - p.ps;
    const int warp = threadIdx.x >> 5;
    if (warp < 2) {
        const uint64_t d = warp ? d1 : d0;
        const uint64_t v = (warp && d1 == p.la + p.lb) ? p.la
                         : warp_merge_split(srcb + p.ps, p.la, srcb + p.ps + p.la, p.lb, d);
        if ((threadIdx.x & 31) == 0) s_split[warp] = v;
    }
    __syncthreads();
    const uint64_t a_s = s_split[0], a_e = s_split[1];
    const uint64_t b_s = d0 - a_s, b_e = d1 - a_e;
    if (!spans_ok(a_s, a_e, b_s, b_e, OT)) {  // CTA-uniform
        if (threadIdx.x == 0) *err = kErrMergeSpan;
        return;
    }
    merge_tile<K, XF>(srcb + p.ps + a_s, (int)(a_e - a_s), srcb + p.ps + p.la + b_s,
                      (int)(b_e - b_s), g.loc(pass) + o, pass == g.P, sm);
}

// Plans and sorts S segments: CSR (`src.offsets`; `count` = elements of the array) or
// descriptors (`count` = sum of the lengths). `max_len` bounds every segment's length.
// The temporaries come from `src` (CSR: aux = base of a count-element buffer).
template <typename K, int XF>
bool seg_sort_keys(Workspace& ws, SegSrc src, uint64_t count, uint64_t S, uint64_t max_len,
                   bool graph) {
    constexpr int TILE = kBlock * SortShape<K>::ITEMS;
    const uint64_t items_cap = S + count / TILE + 1;
    if (items_cap >= 0x7fffffffull) {
        set_error(PARALLAX_ERR_INVALID_ARGUMENT, "segmented sort: too many tiles");
        return false;
    }
    int pass_bound = 0;
    while ((1ull << pass_bound) < (max_len + TILE - 1) / TILE) ++pass_bound;
    auto up = [](size_t v) { return (v + 255) / 256 * 256; };
    const bool csr_tmp = src.offsets != nullptr;
    const size_t tmp_bytes = csr_tmp ? up(count * sizeof(K)) : 0;
    char* t = static_cast<char*>(ws.temp(tmp_bytes + 256));
    char* sb = static_cast<char*>(ws.seg(256 + up((S + 1) * 4) + up(items_cap * 4)));
    // the epoch in counters[2] is shared with the other segmented launches, so a wrap
    // clears their status entries too
    StatusEntry* st = static_cast<StatusEntry*>(ws.seg_status(1));
    if (!t || !sb || !st) return false;
    if (csr_tmp) src.aux = reinterpret_cast<uint64_t>(t);
    src.aux_stride = 0;
    src.elem = sizeof(K);
    uint32_t* counters = reinterpret_cast<uint32_t*>(sb);
    uint32_t* item_start = reinterpret_cast<uint32_t*>(sb + 256);
    uint32_t* item_seg = reinterpret_cast<uint32_t*>(sb + 256 + up((S + 1) * 4));
    ProfScope prof(ws, "segmented_sort", 2 * count * sizeof(K));
    count_launch(3 + pass_bound);
    auto enqueue = [&] {
        cudaStream_t s = ws.stream();
        k_seg_plan<kBlock><<<1, kBlock, 0, s>>>(src, S, count, (uint32_t)TILE, item_start, counters,
                                                SegEmpty::NONE, nullptr, st, ws.seg_status_cap,
                                                &ws.d_slot->spin_error,
                                                items_cap <= kInlineItems ? item_seg : nullptr);
        const unsigned grid = (unsigned)items_cap;
        if (items_cap > kInlineItems)
            k_seg_map<256><<<seg_map_grid(S), 256, 0, s>>>(item_start, S, item_seg);
        k_seg_tile_sort<K, XF><<<grid, kBlock, 0, s>>>(src, S, item_start, item_seg);
        for (int pass = 1; pass <= pass_bound; ++pass)
            k_seg_merge<K, XF><<<grid, kBlock, 0, s>>>(src, S, item_start, item_seg, pass,
                                                       &ws.d_slot->spin_error);
        return cuda_ok(cudaGetLastError(), "segmented sort launch");
    };
    if (!graph) return enqueue();
    char key[256];
    snprintf(key, sizeof key, "segsort/%d/%d/%p/%p/%llu/%llu/%llu", (int)sizeof(K), XF,
             (const void*)src.in, (const void*)src.offsets, (unsigned long long)S,
             (unsigned long long)count, (unsigned long long)max_len);
    return graph_launch(ws, key, enqueue);
}

// by_key (sort_kv records, stable by key) always takes the segmented radix sort; plain keys
// take it when the mean segment spans at least one radix tile, the merge sort otherwise.
bool seg_sort_dispatch(Workspace& ws, DType t, const SegSrc& src, uint64_t count, uint64_t S,
                       uint64_t max_len, bool graph, bool by_key) {
    bool radix = by_key || count / S >= segmented_radix_tile(t);
    if (const char* e = getenv("PARALLAX_SORT")) {
        if (!strcmp(e, "merge") && !by_key) radix = false;
        else if (!strcmp(e, "radix")) radix = true;
    }
    if (radix) return launch_segmented_radix_sort(ws, t, src, count, S, by_key, graph);
    switch (t) {
        case DType::U32: return seg_sort_keys<uint32_t, 0>(ws, src, count, S, max_len, graph);
        case DType::I32: return seg_sort_keys<uint32_t, 1>(ws, src, count, S, max_len, graph);
        case DType::F32: return seg_sort_keys<uint32_t, 2>(ws, src, count, S, max_len, graph);
        case DType::U64: return seg_sort_keys<uint64_t, 0>(ws, src, count, S, max_len, graph);
        case DType::I64: return seg_sort_keys<uint64_t, 1>(ws, src, count, S, max_len, graph);
        case DType::F64: return seg_sort_keys<uint64_t, 2>(ws, src, count, S, max_len, graph);
        default: break;
    }
    set_error(PARALLAX_ERR_INVALID_ARGUMENT, "segmented sort: unsupported element type");
    return false;
}

}  // namespace

// Sizes from which the radix sort (a histogram launch plus one pass per key byte) beats the
// merge sort (a tile-sort launch plus log2(tiles) merge passes). PARALLAX_SORT=merge or
// =radix forces one path (read on every call). Both paths timed on B200 (random keys):
// 4-byte 2^19 radix 0.074 / merge 0.062 ms, 2^20 0.082 / 0.088, 2^21 0.100 / 0.125;
// 8-byte 2^19 0.134 / 0.099 ms, 2^20 0.139 / 0.143, 2^21 0.185 / 0.206.
constexpr size_t kRadixMin4 = size_t(1) << 20;
constexpr size_t kRadixMin8 = size_t(1) << 20;

size_t sort_radix_min(DType t) { return dtype_size(t) == 4 ? kRadixMin4 : kRadixMin8; }

bool launch_sort(Workspace& ws, DType t, void* d_data, size_t n, bool by_key) {
    if (n <= 1) return true;
    // stable by key at every size: only the radix passes over the key bytes give that
    if (by_key) return launch_radix_sort(ws, t, d_data, n, true);
    const size_t es = dtype_size(t);
    bool radix = n >= sort_radix_min(t);
    if (const char* e = getenv("PARALLAX_SORT")) {
        if (!strcmp(e, "merge")) radix = false;
        else if (!strcmp(e, "radix")) radix = true;
    }
    if (radix && (es == 4 || es == 8)) return launch_radix_sort(ws, t, d_data, n);
    switch (t) {
        case DType::U32: return sort_keys<uint32_t, 0>(ws, d_data, n);
        case DType::I32: return sort_keys<uint32_t, 1>(ws, d_data, n);
        case DType::F32: return sort_keys<uint32_t, 2>(ws, d_data, n);
        case DType::U64: return sort_keys<uint64_t, 0>(ws, d_data, n);
        case DType::I64: return sort_keys<uint64_t, 1>(ws, d_data, n);
        case DType::F64: return sort_keys<uint64_t, 2>(ws, d_data, n);
        default: break;
    }
    set_error(PARALLAX_ERR_INVALID_ARGUMENT, "sort: unsupported element type");
    return false;
}

bool launch_segmented_sort_descs(Workspace& ws, DType t, const SegDesc* d_descs, uint64_t S,
                                 uint64_t total, uint64_t max_len, bool by_key) {
    if (S == 0 || total == 0) return true;
    const SegSrc src{nullptr, d_descs, 0, 0, 0, 0, (uint32_t)dtype_size(t)};
    return seg_sort_dispatch(ws, t, src, total, S, max_len, false, by_key);
}

}  // namespace pxb

using namespace pxb;

PXB_EXPORT int parallax_segmented_sort(parallax_kernel_t kernel, void* data, size_t count,
                                       const uint64_t* offsets, size_t num_segments) {
    set_ok();
    Handle* h = as_handle(kernel);
    if (!h || (h->kind != Kind::SORT && h->kind != Kind::SORT_KV)) {
        set_error(PARALLAX_ERR_INVALID_HANDLE, "parallax_segmented_sort: needs a sort or sort_kv handle");
        return PARALLAX_ERR_INVALID_HANDLE;
    }
    Workspace* ws = workspace();
    if (!ws) return PARALLAX_ERR_NO_DEVICE;
    if (num_segments == 0 || count == 0) return PARALLAX_OK;
    void* d = device_operand(data, "parallax_segmented_sort", "data");
    const void* o = d ? device_operand(offsets, "parallax_segmented_sort", "offsets") : nullptr;
    if (!d || !o) return PARALLAX_ERR_INVALID_ARGUMENT;
    const DType t = h->kind == Kind::SORT_KV ? DType::U64 : h->dtype;
    const SegSrc src{static_cast<const uint64_t*>(o), nullptr, reinterpret_cast<uint64_t>(d), 0, 0,
                     0, (uint32_t)dtype_size(t)};
    // CSR: every segment lies within the array, so `count` bounds the longest one
    const bool ok = seg_sort_dispatch(*ws, t, src, count, num_segments, count, true,
                                      h->kind == Kind::SORT_KV);
    if (!ok) return last_error() ? last_error() : PARALLAX_ERR_CUDA;
    return ws->async ? PARALLAX_OK : sync_stream(*ws);
}
