// Single-launch reductions: reduce (sum / max / min), count_if, find, argminmax, mismatch.
//
// Reference: the reduce is an iterative 256-ary shared-memory tree, one dispatch and one
// fence wait per level, one element per thread (src/kernel/kernel_launcher.cpp:908-985,
// shaders/reduce.comp:21-40); argminmax / find / mismatch combine per-block winners on
// the host (kernel_launcher.cpp:1073-1098, :1182-1189, :1273-1277).
//
// Here: one launch. A grid of (resident blocks per SM) x (SM count) threads streams the
// input with 16-byte non-caching loads, UNROLL independent loads in flight per thread,
// folds into per-thread accumulators, reduces warp -> block with shuffles, writes one
// partial per block, and the last block to finish (atomic ticket) folds the partials in
// block order and writes the result. The fold order is a function of n and the grid
// only, so floating-point results are identical from run to run.
#include <float.h>
#include <stdint.h>

#include <limits>
#include <type_traits>

#include "../runtime.hpp"

namespace pxb {
namespace {

constexpr int kBlock = 256;
constexpr int kUnroll = 4;

template <typename T>
struct ArgVal {
    T v;
    uint64_t i;  // UINT64_MAX = empty
};

template <typename T>
__device__ __forceinline__ ArgVal<T> shfl_xor(ArgVal<T> a, int d) {
    ArgVal<T> r;
    r.v = __shfl_xor_sync(0xffffffffu, a.v, d);
    r.i = __shfl_xor_sync(0xffffffffu, (unsigned long long)a.i, d);
    return r;
}
using pxb::shfl_xor;

template <typename A, typename Op>
__device__ __forceinline__ A warp_fold(A v, Op op) {
#pragma unroll
    for (int d = 16; d >= 1; d >>= 1) v = op(v, shfl_xor(v, d));
    return v;
}

// Block-wide fold; the result is valid in thread 0. Callers separate two uses with a
// __syncthreads().
template <typename A, typename Op>
__device__ __forceinline__ A block_fold(A v, Op op, A ident) {
    __shared__ A s[kBlock / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    v = warp_fold(v, op);
    if (lane == 0) s[warp] = v;
    __syncthreads();
    if (warp == 0) {
        v = lane < kBlock / 32 ? s[lane] : ident;
        v = warp_fold(v, op);
    }
    return v;
}

// ---- element transforms: (x, index) -> accumulator -------------------------------------
template <typename T, typename A>
struct XfValue {
    __device__ __forceinline__ A operator()(T x, uint64_t) const { return (A)x; }
};

template <typename T>
struct PredEval {
    PredKind kind;
    bool negate;
    T c;
    T m, r;
    FastMod32 fm;  // 32-bit element types: m as an invariant divisor
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
            case PredKind::MOD: v = mod_eq(x); break;
            default: v = false; break;
        }
        return v != negate;
    }
    template <typename U = T>
    __device__ __forceinline__ bool mod_eq(U x) const {
        if constexpr (std::is_integral<U>::value && sizeof(U) == 4) return fm.eq(x, r);
        else if constexpr (std::is_integral<U>::value)  // x % -1 == 0 (no overflowing division)
            return (std::is_signed<U>::value && m == U(-1)) ? r == U(0) : x % m == r;
        else return false;
    }
};

template <typename T>
struct XfCount {
    PredEval<T> p;
    __device__ __forceinline__ unsigned long long operator()(T x, uint64_t) const {
        return p(x) ? 1ull : 0ull;
    }
};
template <typename T>
struct XfFind {
    PredEval<T> p;
    __device__ __forceinline__ unsigned long long operator()(T x, uint64_t i) const {
        return p(x) ? (unsigned long long)i : ~0ull;
    }
};
template <typename T>
struct XfArg {
    __device__ __forceinline__ ArgVal<T> operator()(T x, uint64_t i) const { return {x, i}; }
};

struct OpMinU64 {
    __device__ __forceinline__ unsigned long long operator()(unsigned long long a,
                                                             unsigned long long b) const {
        return b < a ? b : a;
    }
};

// First (or last) minimum / maximum; empty slots lose.
template <typename T>
struct OpArg {
    bool want_max, want_last;
    __device__ __forceinline__ ArgVal<T> operator()(ArgVal<T> a, ArgVal<T> b) const {
        if (a.i == ~0ull) return b;
        if (b.i == ~0ull) return a;
        bool b_better = want_max ? (b.v > a.v) : (b.v < a.v);
        bool a_better = want_max ? (a.v > b.v) : (a.v < b.v);
        if (b_better) return b;
        if (a_better) return a;
        // equal (or unordered): index decides
        return want_last ? (b.i > a.i ? b : a) : (b.i < a.i ? b : a);
    }
};

template <typename A>
__device__ __forceinline__ void store_result(A* out, A v) { *out = v; }

// ---- the kernel -----------------------------------------------------------------------------
// in: n elements, the first `head` of which precede the first 16-byte boundary.
template <typename T, typename A, typename R, typename Xf, typename Op>
__global__ void __launch_bounds__(kBlock)
k_reduce(const T* __restrict__ in, uint64_t n, uint64_t head, Xf xf, Op op, A ident,
         A* __restrict__ partials, unsigned* __restrict__ ticket, R* __restrict__ out) {
    constexpr int V = 16 / sizeof(T);
    const uint64_t G = (uint64_t)gridDim.x * kBlock;
    const uint64_t g = (uint64_t)blockIdx.x * kBlock + threadIdx.x;
    A acc[kUnroll];
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) acc[u] = ident;

    const uint64_t nv = (n - head) / V;
    const uint4* vp = reinterpret_cast<const uint4*>(in + head);
    uint64_t i = g;
    for (; i + (kUnroll - 1) * G < nv; i += kUnroll * G) {
        uint4 r[kUnroll];
#pragma unroll
        for (int u = 0; u < kUnroll; ++u) r[u] = ldg_stream16(vp + i + u * G);
#pragma unroll
        for (int u = 0; u < kUnroll; ++u) {
            const T* e = reinterpret_cast<const T*>(&r[u]);
            const uint64_t base = head + (i + u * G) * V;
#pragma unroll
            for (int k = 0; k < V; ++k) acc[u] = op(acc[u], xf(e[k], base + k));
        }
    }
    for (; i < nv; i += G) {
        uint4 r = ldg_stream16(vp + i);
        const T* e = reinterpret_cast<const T*>(&r);
        const uint64_t base = head + i * V;
#pragma unroll
        for (int k = 0; k < V; ++k) acc[0] = op(acc[0], xf(e[k], base + k));
    }
    const uint64_t tail0 = head + nv * V;
    for (uint64_t j = g; j < head; j += G) acc[0] = op(acc[0], xf(in[j], j));
    if (g < n - tail0) acc[kUnroll - 1] = op(acc[kUnroll - 1], xf(in[tail0 + g], tail0 + g));
    A a = acc[0];
#pragma unroll
    for (int u = 1; u < kUnroll; ++u) a = op(a, acc[u]);

    a = block_fold(a, op, ident);
    __shared__ bool s_last;
    if (threadIdx.x == 0) {
        partials[blockIdx.x] = a;
        __threadfence();
        unsigned t = atomicAdd(ticket, 1u);
        s_last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    A b = ident;
    for (unsigned j = threadIdx.x; j < gridDim.x; j += kBlock)
        b = op(b, *reinterpret_cast<volatile A*>(partials + j));
    b = block_fold(b, op, ident);
    if (threadIdx.x == 0) {
        store_result(out, (R)b);
        *ticket = 0;  // self-reset for the next launch on this workspace
    }
}

// ArgVal -> index result
template <typename T>
struct ArgToIndex {
    uint64_t v;
    __device__ ArgToIndex(ArgVal<T> a) : v(a.i == ~0ull ? 0ull : a.i) {}
};

template <typename K>
int grid_for(K kernel, uint64_t nvec) {
    static int per_sm = 0;
    if (!per_sm) {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kBlock, 0);
        if (per_sm <= 0) per_sm = 1;
    }
    uint64_t max_blocks = (uint64_t)per_sm * device_info().sm_count;
    uint64_t want = (nvec + (uint64_t)kBlock * kUnroll - 1) / ((uint64_t)kBlock * kUnroll);
    if (want < 1) want = 1;
    return (int)(want < max_blocks ? want : max_blocks);
}

template <typename T>
uint64_t head_of(const void* p, uint64_t n) {
    uintptr_t a = reinterpret_cast<uintptr_t>(p);
    if (a % sizeof(T)) return n;  // misaligned element pointer: scalar path only
    uint64_t h = ((16 - (a % 16)) % 16) / sizeof(T);
    return h < n ? h : n;
}

// Ticket and partials live in the small scratch region (ScratchOff).
template <typename T, typename A, typename R, typename Xf, typename Op>
bool run(Workspace& ws, const char* name, const void* d_in, uint64_t n, Xf xf, Op op, A ident,
         R* d_out) {
    auto kernel = k_reduce<T, A, R, Xf, Op>;
    uint64_t head = head_of<T>(d_in, n);
    uint64_t nvec = (n - head) / (16 / sizeof(T));
    int grid = grid_for(kernel, nvec);
    constexpr size_t kMaxPartials = (kScratchSmall - ScratchOff::partials) / sizeof(A);
    if ((size_t)grid > kMaxPartials) grid = (int)kMaxPartials;
    char* scratch = ws.scratch(0);
    if (!scratch) return false;
    unsigned* ticket = reinterpret_cast<unsigned*>(scratch + ScratchOff::ticket);
    A* partials = reinterpret_cast<A*>(scratch + ScratchOff::partials);
    {
        ProfScope prof(ws, name, n * sizeof(T));
        kernel<<<grid, kBlock, 0, ws.stream()>>>(static_cast<const T*>(d_in), n, head, xf, op,
                                                 ident, partials, ticket, d_out);
    }
    count_launch();
    return cuda_ok(cudaGetLastError(), "k_reduce launch");
}

template <typename T>
PredEval<T> make_pred(const Pred& p) {
    PredEval<T> e;
    e.kind = p.kind;
    e.negate = p.negate;
    if (std::is_floating_point<T>::value) e.c = (T)p.f;
    else if (std::is_signed<T>::value) e.c = (T)p.i;
    else e.c = (T)p.u;
    e.m = (T)p.mod_m;
    e.r = (T)p.mod_r;
    if (std::is_integral<T>::value && sizeof(T) == 4) e.fm = FastMod32::make((int64_t)e.m);
    return e;
}

template <typename T>
bool reduce_typed(Workspace& ws, RedOp op, const void* d_in, uint64_t n, void* d_out) {
    T* out = static_cast<T*>(d_out);
    if (op == RedOp::SUM) {
        using A = typename SumAcc<T>::type;
        return run<T, A, T>(ws, "k_reduce_sum", d_in, n, XfValue<T, A>{}, OpSum{}, A(0), out);
    }
    if (op == RedOp::MAX) {
        T ident = std::numeric_limits<T>::has_infinity ? -std::numeric_limits<T>::infinity()
                                                       : std::numeric_limits<T>::lowest();
        return run<T, T, T>(ws, "k_reduce_max", d_in, n, XfValue<T, T>{}, OpMax{}, ident, out);
    }
    T ident = std::numeric_limits<T>::has_infinity ? std::numeric_limits<T>::infinity()
                                                   : std::numeric_limits<T>::max();
    return run<T, T, T>(ws, "k_reduce_min", d_in, n, XfValue<T, T>{}, OpMin{}, ident, out);
}

struct XfNonzeroByte {
    __device__ __forceinline__ unsigned long long operator()(uint8_t x, uint64_t) const {
        return x != 0 ? 1ull : 0ull;
    }
};

template <typename T>
bool count_typed(Workspace& ws, const Pred& p, const void* d_in, uint64_t n, uint64_t* d_out) {
    return run<T, unsigned long long, unsigned long long>(
        ws, "k_count_if", d_in, n, XfCount<T>{make_pred<T>(p)}, OpSum{}, 0ull,
        reinterpret_cast<unsigned long long*>(d_out));
}

template <typename T>
bool find_typed(Workspace& ws, const Pred& p, const void* d_in, uint64_t n, uint64_t* d_out) {
    // Non-matching elements map to ~0; seeding the min-fold with n reports "not found"
    // as n.
    return run<T, unsigned long long, unsigned long long>(
        ws, "k_find", d_in, n, XfFind<T>{make_pred<T>(p)}, OpMinU64{}, (unsigned long long)n,
        reinterpret_cast<unsigned long long*>(d_out));
}

template <typename T>
bool argminmax_typed(Workspace& ws, bool want_max, bool want_last, const void* d_in,
                     uint64_t n, uint64_t* d_out) {
    ArgVal<T> ident{T(0), ~0ull};
    return run<T, ArgVal<T>, ArgToIndex<T>>(ws, "k_argminmax", d_in, n, XfArg<T>{}, OpArg<T>{want_max, want_last},
                                            ident, reinterpret_cast<ArgToIndex<T>*>(d_out));
}

// ---- mismatch: first i with a[i] != b[i] ------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(kBlock)
k_mismatch(const T* __restrict__ a, const T* __restrict__ b, uint64_t n, bool vec_ok,
           unsigned long long* __restrict__ partials, unsigned* __restrict__ ticket,
           unsigned long long* __restrict__ out) {
    constexpr int V = 16 / sizeof(T);
    const uint64_t G = (uint64_t)gridDim.x * kBlock;
    const uint64_t g = (uint64_t)blockIdx.x * kBlock + threadIdx.x;
    unsigned long long best = n;
    uint64_t done = 0;
    if (vec_ok) {
        const uint64_t nv = n / V;
        const uint4* va = reinterpret_cast<const uint4*>(a);
        const uint4* vb = reinterpret_cast<const uint4*>(b);
        for (uint64_t i = g; i < nv; i += G) {
            uint4 x = ldg_stream16(va + i), y = ldg_stream16(vb + i);
            const T* ex = reinterpret_cast<const T*>(&x);
            const T* ey = reinterpret_cast<const T*>(&y);
#pragma unroll
            for (int k = 0; k < V; ++k)
                if (!(ex[k] == ey[k]) && i * V + k < best) best = i * V + k;
        }
        done = nv * V;
    }
    for (uint64_t i = done + g; i < n; i += G)
        if (!(a[i] == b[i]) && i < best) best = i;
    OpMinU64 op;
    best = block_fold(best, op, (unsigned long long)n);
    __shared__ bool s_last;
    if (threadIdx.x == 0) {
        partials[blockIdx.x] = best;
        __threadfence();
        s_last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    unsigned long long m = n;
    for (unsigned j = threadIdx.x; j < gridDim.x; j += kBlock)
        m = op(m, *reinterpret_cast<volatile unsigned long long*>(partials + j));
    m = block_fold(m, op, (unsigned long long)n);
    if (threadIdx.x == 0) {
        *out = m;
        *ticket = 0;
    }
}

template <typename T>
bool mismatch_typed(Workspace& ws, const void* a, const void* b, uint64_t n, uint64_t* d_out) {
    auto kernel = k_mismatch<T>;
    uintptr_t pa = reinterpret_cast<uintptr_t>(a), pb = reinterpret_cast<uintptr_t>(b);
    bool vec_ok = (pa % 16 == 0) && (pb % 16 == 0);
    int grid = grid_for(kernel, n / (16 / sizeof(T)));
    constexpr size_t kMaxPartials = (kScratchSmall - ScratchOff::partials) / 8;
    if ((size_t)grid > kMaxPartials) grid = (int)kMaxPartials;
    char* scratch = ws.scratch(0);
    if (!scratch) return false;
    {
        ProfScope prof(ws, "k_mismatch", 2 * n * sizeof(T));
        kernel<<<grid, kBlock, 0, ws.stream()>>>(
            static_cast<const T*>(a), static_cast<const T*>(b), n, vec_ok,
            reinterpret_cast<unsigned long long*>(scratch + ScratchOff::partials),
            reinterpret_cast<unsigned*>(scratch + ScratchOff::ticket),
            reinterpret_cast<unsigned long long*>(d_out));
    }
    count_launch();
    return cuda_ok(cudaGetLastError(), "k_mismatch launch");
}

#define PXB_DISPATCH(t, CALL)                                     \
    switch (t) {                                                  \
        case DType::F32: { using T = float; return CALL; }        \
        case DType::F64: { using T = double; return CALL; }       \
        case DType::I32: { using T = int32_t; return CALL; }      \
        case DType::I64: { using T = int64_t; return CALL; }      \
        case DType::U32: { using T = uint32_t; return CALL; }     \
        case DType::U64: { using T = uint64_t; return CALL; }     \
        default: break;                                           \
    }

}  // namespace

bool launch_reduce(Workspace& ws, DType t, RedOp op, const void* d_in, size_t n, void* d_out) {
    PXB_DISPATCH(t, reduce_typed<T>(ws, op, d_in, n, d_out));
    set_error(PARALLAX_ERR_INVALID_ARGUMENT, "reduce: unsupported element type");
    return false;
}
bool launch_count_if(Workspace& ws, DType t, const Pred& p, const void* d_in, size_t n,
                     uint64_t* d_count) {
    PXB_DISPATCH(t, count_typed<T>(ws, p, d_in, n, d_count));
    set_error(PARALLAX_ERR_INVALID_ARGUMENT, "count_if: unsupported element type");
    return false;
}
bool launch_find(Workspace& ws, DType t, const Pred& p, const void* d_in, size_t n,
                 uint64_t* d_index) {
    PXB_DISPATCH(t, find_typed<T>(ws, p, d_in, n, d_index));
    set_error(PARALLAX_ERR_INVALID_ARGUMENT, "find: unsupported element type");
    return false;
}
bool launch_argminmax(Workspace& ws, DType t, bool want_max, bool want_last, const void* d_in,
                      size_t n, uint64_t* d_index) {
    PXB_DISPATCH(t, argminmax_typed<T>(ws, want_max, want_last, d_in, n, d_index));
    set_error(PARALLAX_ERR_INVALID_ARGUMENT, "argminmax: unsupported element type");
    return false;
}
bool launch_mismatch(Workspace& ws, DType t, const void* d_a, const void* d_b, size_t n,
                     uint64_t* d_index) {
    PXB_DISPATCH(t, mismatch_typed<T>(ws, d_a, d_b, n, d_index));
    set_error(PARALLAX_ERR_INVALID_ARGUMENT, "mismatch: unsupported element type");
    return false;
}

bool launch_count_flags(Workspace& ws, const uint8_t* d_flags, size_t n, uint64_t* d_count) {
    return run<uint8_t, unsigned long long, unsigned long long>(
        ws, "k_count_flags", d_flags, n, XfNonzeroByte{}, OpSum{}, 0ull,
        reinterpret_cast<unsigned long long*>(d_count));
}

}  // namespace pxb
