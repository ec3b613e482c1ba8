// Single-pass inclusive / exclusive '+' scan.
//
// Reference: block Hillis-Steele scan (8 rounds, 2 barriers each) + recursive scan of the
// block sums + an add-offsets pass, each a separate dispatch with a fence wait
// (src/kernel/kernel_launcher.cpp:1280-1342, shaders/scan.comp:16-35,
// shaders/scan_add.comp:14-19); exclusive adds a shift pass writing
// out[i] = init + incl[i-1] (kernel_launcher.cpp:1346-1475).
//
// Here: one launch, one CTA per tile, in blockIdx order. Each CTA
//   1. stages its tile (256 threads x 3 x 16 bytes = 12 KiB) in shared memory with one
//      bulk copy (cp.async.bulk + mbarrier),
//   2. scans 12 (4-byte) or 6 (8-byte) consecutive elements per thread in registers
//      (rows of 48 bytes: conflict-free 128-bit shared loads),
//   3. scans thread totals with warp shuffles and warp totals in one warp,
//   4. gets the tile's exclusive prefix by decoupled look-back (lookback.cuh),
//   5. writes results into the staged tile and stores it with one bulk copy.
// HBM traffic is the algorithmic minimum: n*s read + n*s written.
// Accumulation: fp32 data is scanned per thread in fp32 (12 terms) and carried across
// threads, warps and tiles in fp64; integers wrap around in their unsigned type.
#include <stdint.h>
#include <string.h>

#include <mutex>

#include "../lookback.cuh"
#include "../runtime.hpp"
#include "../tma.cuh"

namespace pxb {
namespace {

constexpr int kBlock = 256;
constexpr int kVpt = 3;  // 16-byte vectors per thread; odd => conflict-free row reads

template <typename T> struct ScanTypes;
template <> struct ScanTypes<float> { using L = float; using A = double; };
template <> struct ScanTypes<double> { using L = double; using A = double; };
template <> struct ScanTypes<int32_t> { using L = uint32_t; using A = uint32_t; };
template <> struct ScanTypes<uint32_t> { using L = uint32_t; using A = uint32_t; };
template <> struct ScanTypes<int64_t> { using L = uint64_t; using A = uint64_t; };
template <> struct ScanTypes<uint64_t> { using L = uint64_t; using A = uint64_t; };

template <typename T>
struct ScanShape {
    static constexpr int V = 16 / sizeof(T);
    static constexpr int ITEMS = kVpt * V;
    static constexpr int TILE = kBlock * ITEMS;
};

template <typename T, bool EXCL, bool BULK>
__global__ void __launch_bounds__(kBlock)
k_scan(const T* in, T* out, uint64_t n,  // in == out allowed (in-place ABI scan)
       typename ScanTypes<T>::A init, TileStatus<typename ScanTypes<T>::A> ts) {
    using L = typename ScanTypes<T>::L;
    using A = typename ScanTypes<T>::A;
    constexpr int V = ScanShape<T>::V;
    constexpr int ITEMS = ScanShape<T>::ITEMS;
    constexpr int TILE = ScanShape<T>::TILE;
    __shared__ __align__(128) T buf[TILE];
    __shared__ __align__(8) uint64_t bar;
    __shared__ A s_warp[kBlock / 32];

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint64_t tile = blockIdx.x;
    const uint64_t base = tile * (uint64_t)TILE;
    const uint64_t rem = n - base;
    const uint32_t cnt = rem < (uint64_t)TILE ? (uint32_t)rem : (uint32_t)TILE;

    uint32_t bulk = 0;  // elements moved by the bulk copies
    if constexpr (BULK) {
        bulk = (uint32_t)((cnt * sizeof(T)) / 16 * 16 / sizeof(T));
        if (tid == 0) {
            mbar_init(&bar, 1);
            fence_mbar_init();
            mbar_arrive_expect_tx(&bar, bulk * (uint32_t)sizeof(T));
            if (bulk) bulk_load(buf, in + base, bulk * (uint32_t)sizeof(T), &bar);
        }
    }
    // ragged end of the last tile (and everything when not bulk-aligned): plain loads
    for (uint32_t e = bulk + tid; e < (uint32_t)TILE; e += kBlock)
        buf[e] = e < cnt ? in[base + e] : T(0);
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

    // ---- per-thread scan of ITEMS consecutive elements ----
    L x[ITEMS];
    {
        const uint4* row = reinterpret_cast<const uint4*>(buf + tid * ITEMS);
#pragma unroll
        for (int v = 0; v < kVpt; ++v) {
            uint4 r = row[v];
            const T* e = reinterpret_cast<const T*>(&r);
#pragma unroll
            for (int k = 0; k < V; ++k) x[v * V + k] = (L)e[k];
        }
    }
#pragma unroll
    for (int j = 1; j < ITEMS; ++j) x[j] = x[j - 1] + x[j];

    // ---- warp and block scan of thread totals ----
    const A tot = (A)x[ITEMS - 1];
    const A incl = warp_inclusive_scan(tot, OpSum());
    A texcl = shfl_up(incl, 1);
    if (lane == 0) texcl = A(0);
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        const A w = lane < kBlock / 32 ? s_warp[lane] : A(0);
        const A wi = warp_inclusive_scan(w, OpSum());
        const A agg = shfl_idx(wi, kBlock / 32 - 1);
        A wex = shfl_up(wi, 1);
        if (lane == 0) wex = A(0);
        const A prefix = lookback(ts, tile, agg);
        if (lane < kBlock / 32) s_warp[lane] = prefix + wex;
    }
    __syncthreads();
    A tb = s_warp[warp] + texcl;
    if constexpr (EXCL) tb = init + tb;

    // ---- results back into the staged tile ----
    {
        uint4* row = reinterpret_cast<uint4*>(buf + tid * ITEMS);
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
    }
    if constexpr (BULK) fence_proxy_async_smem();
    __syncthreads();
    if constexpr (BULK) {
        if (tid == 0 && bulk) {
            bulk_store(out + base, buf, bulk * (uint32_t)sizeof(T));
            bulk_commit();
        }
    }
    for (uint32_t e = bulk + tid; e < cnt; e += kBlock) out[base + e] = buf[e];
    if constexpr (BULK) {
        if (tid == 0 && bulk) bulk_wait_all();
    }
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
    const bool bulk = (reinterpret_cast<uintptr_t>(d_in) % 16 == 0) &&
                      (reinterpret_cast<uintptr_t>(d_out) % 16 == 0);
    const T* in = static_cast<const T*>(d_in);
    T* out = static_cast<T*>(d_out);
    dim3 grid((unsigned)tiles);
    cudaStream_t s = ws.stream();
    ProfScope prof(ws, exclusive ? "k_scan_exclusive" : "k_scan_inclusive", 2 * n * sizeof(T));
    if (exclusive) {
        if (bulk) k_scan<T, true, true><<<grid, kBlock, 0, s>>>(in, out, n, init, ts);
        else k_scan<T, true, false><<<grid, kBlock, 0, s>>>(in, out, n, init, ts);
    } else {
        if (bulk) k_scan<T, false, true><<<grid, kBlock, 0, s>>>(in, out, n, init, ts);
        else k_scan<T, false, false><<<grid, kBlock, 0, s>>>(in, out, n, init, ts);
    }
    count_launch();
    return cuda_ok(cudaGetLastError(), "k_scan launch");
}

}  // namespace

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

}  // namespace pxb

// ---- allocation-free scan -----------------------------------------------------------------
// Some callers cannot allocate device memory at all: code that runs inside an allocation
// hook (a malloc / operator new interposer that routes the heap into the arena would
// re-enter itself if the runtime allocated), or a process whose device memory has been
// handed to its own pool. parallax_scan_noalloc gives them the single-pass scan with no
// allocation by the runtime: the look-back status lives in the fixed static device array
// below (576.25 KiB, held on every GPU that loads this library until the process exits),
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
    dim3 grid((unsigned)tiles);
    if (init_host) {
        if (bulk) k_scan<T, true, true><<<grid, kBlock, 0, s>>>(in, out, n, init, ts);
        else k_scan<T, true, false><<<grid, kBlock, 0, s>>>(in, out, n, init, ts);
    } else {
        if (bulk) k_scan<T, false, true><<<grid, kBlock, 0, s>>>(in, out, n, init, ts);
        else k_scan<T, false, false><<<grid, kBlock, 0, s>>>(in, out, n, init, ts);
    }
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
