// Device-resident arena with a pinned host mirror.
//
// Replaces the reference UnifiedArena (src/memory/arena.cpp:21-181, :336-406 and the C
// accessors in src/memory/unified_allocator.cpp:55-103). The reference maps one Vulkan
// buffer into the host (UMA) or keeps a device buffer plus a staging copy and moves the
// WHOLE used range both ways around every top-level call (arena.cpp:296-304). Here:
//   * device side: one contiguous virtual range (cuMemAddressReserve) whose physical
//     HBM is mapped in 512 MiB chunks as the arena grows, so a 64 GiB capacity costs
//     nothing until used;
//   * host side: one contiguous anonymous mapping of the same size; a chunk's pages are
//     locked the first time a copy touches it (host<->device copies then run at full
//     link speed), so device-resident blocks cost no host memory;
//   * the relocation formula of the reference stays exact: the device address of a
//     host arena pointer p is dev_base + (p - host_base);
//   * blocks carry a residency mode; ABI calls move only the byte ranges they name
//     (see abi.cu), never the whole arena;
//   * allocation is first-fit over an offset-ordered free map with coalescing (the
//     reference never coalesces, arena.cpp:354-355), 256-byte minimum alignment.
// Pool-backed mode (whole-heap capture; reference arena.cpp:183-275, :336-386): when the
// heap pool (heap_pool.cu) is live at the arena's first use - a program linked with the
// capture shim lib/libparallax-heap.a, or one that called px_pool_init() - the arena adopts
// the pool's reservation instead of mapping memory of its own, and works like the
// reference's imported host memory: the pool is page-locked (cudaHostRegister) in 64 MiB
// chunks up to its high-water mark before any kernel that may touch it runs, its device
// address is its host address (dev_base == host_base, so stored heap pointers relocate to
// themselves), and kernels read and write it in place over the host link. Nothing is
// copied, so no copy can ever overwrite a host-side change, and every heap pointer is an
// arena pointer. Arena blocks are pool blocks (px_pool_alloc); residency modes and the
// explicit sync calls have nothing to do in this mode. Needs a device that can use host
// pointers for registered memory (a range that cannot be registered is still usable on a
// device with pageable-memory access); otherwise the arena keeps its own mapping.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/mman.h>

#include <map>
#include <mutex>
#include <vector>

#include "parallax/heap_pool.h"
#include "runtime.hpp"

namespace pxb {

namespace {

constexpr size_t kAlign = 256;
constexpr size_t kDefaultCapacityMiB = 64 * 1024;  // 64 GiB of address space

struct DriverFns {
    PFN_cuMemAddressReserve reserve = nullptr;
    PFN_cuMemCreate create = nullptr;
    PFN_cuMemMap map = nullptr;
    PFN_cuMemSetAccess set_access = nullptr;
    PFN_cuMemGetAllocationGranularity granularity = nullptr;
    bool load() {
        cudaDriverEntryPointQueryResult q;
        auto get = [&](const char* name, void** fn) {
            return cudaGetDriverEntryPoint(name, fn, cudaEnableDefault, &q) == cudaSuccess &&
                   q == cudaDriverEntryPointSuccess && *fn;
        };
        return get("cuMemAddressReserve", (void**)&reserve) &&
               get("cuMemCreate", (void**)&create) && get("cuMemMap", (void**)&map) &&
               get("cuMemSetAccess", (void**)&set_access) &&
               get("cuMemGetAllocationGranularity", (void**)&granularity);
    }
};

struct Arena {
    std::mutex mu;
    bool tried = false;
    bool ok = false;
    bool pool = false;     // pool-backed: zero-copy over the heap pool's reservation
    bool pageable = false;   // the device reaches pageable host memory itself (HMM)
    size_t pool_locked = 0;  // pool bytes page-locked so far (from the base)
    size_t capacity = 0;
    char* host_base = nullptr;
    CUdeviceptr dev_base = 0;
    size_t chunk = 512ull << 20;
    size_t mapped = 0;     // bytes with device memory mapped
    size_t bump = 0;       // first never-used offset
    size_t used = 0;       // bytes in live blocks
    std::map<size_t, size_t> free_blocks;       // offset -> size, coalesced
    std::map<size_t, ArenaBlock> live;          // offset -> block
    DriverFns drv;
    std::vector<CUmemGenericAllocationHandle> handles;
    std::vector<uint8_t> pinned;  // per chunk: host mirror page-locked yet
    bool host_ptr_ok = false;     // kernels may use registered host addresses as they are

    // pin_range, then whether every chunk of the range is page-locked
    bool pinned_range(size_t off, size_t bytes) {
        pin_range(off, bytes);
        std::lock_guard<std::mutex> g(mu);
        for (size_t c = off / chunk; c * chunk < off + bytes; ++c)
            if (c >= pinned.size() || !pinned[c]) return false;
        return true;
    }

    // Page-locks the host mirror of every chunk that [off, off + bytes) touches, on first
    // use: blocks that only ever live on the device never pin host memory.
    void pin_range(size_t off, size_t bytes) {
        std::lock_guard<std::mutex> g(mu);
        for (size_t c = off / chunk; c * chunk < off + bytes && c < pinned.size(); ++c) {
            if (pinned[c]) continue;
            // the pool's reservation may end inside its last chunk
            const size_t len = capacity - c * chunk < chunk ? capacity - c * chunk : chunk;
            if (cudaHostRegister(host_base + c * chunk, len, cudaHostRegisterDefault) !=
                cudaSuccess) {
                cudaGetLastError();  // copies from this chunk stay pageable (slower, correct)
                continue;
            }
            pinned[c] = 1;
        }
    }

    static size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

    bool init() {
        if (tried) return ok;
        tried = true;
        if (!ensure_device()) return false;
        size_t mib = kDefaultCapacityMiB;
        if (const char* e = getenv("PARALLAX_ARENA_SIZE")) {
            unsigned long long v = strtoull(e, nullptr, 10);
            if (v > 0) mib = v;
        }
        size_t free_b = 0, total_b = 0;
        cudaMemGetInfo(&free_b, &total_b);
        capacity = mib << 20;
        if (total_b && capacity > total_b / 10 * 9) capacity = total_b / 10 * 9;
        if (!drv.load()) {
            set_error(PARALLAX_ERR_CUDA, "arena: CUDA virtual memory entry points unavailable");
            return false;
        }
        CUmemAllocationProp prop{};
        prop.type = CU_MEM_ALLOCATION_TYPE_PINNED;
        prop.location.type = CU_MEM_LOCATION_TYPE_DEVICE;
        prop.location.id = device_info().device;
        size_t gran = 0;
        if (drv.granularity(&gran, &prop, CU_MEM_ALLOC_GRANULARITY_RECOMMENDED) != CUDA_SUCCESS ||
            gran == 0)
            gran = 2ull << 20;
        chunk = align_up(chunk, gran);
        capacity = align_up(capacity, chunk);
        int host_ptrs = 0;
        cudaDeviceGetAttribute(&host_ptrs, cudaDevAttrCanUseHostPointerForRegisteredMem,
                               device_info().device);
        host_ptr_ok = host_ptrs != 0;
        void* pb = heap_pool_base();
        if (pb && host_ptrs) {  // whole-heap capture: adopt the pool, zero-copy
            pool = true;
            int pma = 0;
            cudaDeviceGetAttribute(&pma, cudaDevAttrPageableMemoryAccess, device_info().device);
            pageable = pma != 0;
            capacity = heap_pool_reservation();
            host_base = static_cast<char*>(pb);
            dev_base = reinterpret_cast<CUdeviceptr>(pb);
            ok = true;
            if (getenv("PARALLAX_DEBUG"))
                fprintf(stderr, "[parallax] arena: pool-backed, %zu MiB host_base=%p dev_base=0x%llx\n",
                        capacity >> 20, (void*)host_base, (unsigned long long)dev_base);
            return true;
        }
        if (drv.reserve(&dev_base, capacity, chunk, 0, 0) != CUDA_SUCCESS) {
            set_error(PARALLAX_ERR_OUT_OF_MEMORY, "arena: cannot reserve %zu MiB of device VA",
                      capacity >> 20);
            return false;
        }
        void* h = mmap(nullptr, capacity, PROT_READ | PROT_WRITE,
                       MAP_PRIVATE | MAP_ANONYMOUS | MAP_NORESERVE, -1, 0);
        if (h == MAP_FAILED) {
            set_error(PARALLAX_ERR_OUT_OF_MEMORY, "arena: cannot reserve %zu MiB of host VA",
                      capacity >> 20);
            return false;
        }
        host_base = static_cast<char*>(h);
        ok = true;
        if (getenv("PARALLAX_DEBUG"))
            fprintf(stderr, "[parallax] arena: capacity %zu MiB host_base=%p dev_base=0x%llx\n",
                    capacity >> 20, (void*)host_base, (unsigned long long)dev_base);
        return true;
    }

    // Maps device memory (and locks the host mirror) up to `end` bytes.
    bool grow_to(size_t end) {
        while (mapped < end) {
            CUmemAllocationProp prop{};
            prop.type = CU_MEM_ALLOCATION_TYPE_PINNED;
            prop.location.type = CU_MEM_LOCATION_TYPE_DEVICE;
            prop.location.id = device_info().device;
            CUmemGenericAllocationHandle hdl;
            if (drv.create(&hdl, chunk, &prop, 0) != CUDA_SUCCESS) return false;
            if (drv.map(dev_base + mapped, chunk, 0, hdl, 0) != CUDA_SUCCESS) return false;
            CUmemAccessDesc acc{};
            acc.location = prop.location;
            acc.flags = CU_MEM_ACCESS_FLAGS_PROT_READWRITE;
            if (drv.set_access(dev_base + mapped, chunk, &acc, 1) != CUDA_SUCCESS) return false;
            handles.push_back(hdl);
            pinned.push_back(0);
            mapped += chunk;
        }
        return true;
    }

    void* allocate(size_t size, size_t align) {
        if (size == 0) return nullptr;
        std::lock_guard<std::mutex> g(mu);
        if (!init()) return nullptr;
        size_t a = align < kAlign ? kAlign : align;
        if (a & (a - 1)) a = align_up(a, kAlign);
        size_t need = align_up(size, kAlign);
        if (pool) {
            char* p = static_cast<char*>(px_pool_alloc(need, a));
            if (!p) {
                set_error(PARALLAX_ERR_OUT_OF_MEMORY, "arena: heap pool exhausted (%zu bytes)", need);
                return nullptr;
            }
            return commit((size_t)(p - host_base), need);
        }
        // first fit in offset order (a best-fit index by size, measured on the serving mix of
        // small requests with hundreds of blocks live, made allocation-heavy clients ~10 %
        // slower: the first fitting range is usually among the first few)
        for (auto it = free_blocks.begin(); it != free_blocks.end(); ++it) {
            size_t off = align_up(it->first, a);
            size_t pad = off - it->first;
            if (it->second < pad + need) continue;
            size_t blk_off = it->first, blk_size = it->second;
            free_blocks.erase(it);
            if (pad) free_blocks[blk_off] = pad;
            size_t rest = blk_size - pad - need;
            if (rest) free_blocks[off + need] = rest;
            return commit(off, need);
        }
        size_t off = align_up(bump, a);
        if (off + need > capacity) {
            set_error(PARALLAX_ERR_OUT_OF_MEMORY,
                      "arena: out of memory (requested %zu bytes, %zu of %zu in use)", need, used,
                      capacity);
            return nullptr;
        }
        if (!grow_to(off + need)) {
            set_error(PARALLAX_ERR_OUT_OF_MEMORY, "arena: cannot map device memory for %zu bytes",
                      need);
            return nullptr;
        }
        if (off > bump) free_blocks[bump] = off - bump;
        bump = off + need;
        return commit(off, need);
    }

    void* commit(size_t off, size_t need) {
        ArenaBlock b;
        b.offset = off;
        b.size = need;
        b.residency = PARALLAX_COHERENT;
        live[off] = b;
        used += need;
        return host_base + off;
    }

    void deallocate(void* p) {
        if (!p) return;
        std::lock_guard<std::mutex> g(mu);
        if (!ok || !contains(p)) return;
        size_t off = static_cast<char*>(p) - host_base;
        auto it = live.find(off);
        if (it == live.end()) return;  // not a block start or double free: ignore
        size_t size = it->second.size;
        live.erase(it);
        used -= size;
        if (pool) {
            px_pool_free(p);
            return;
        }
        // insert and coalesce with neighbours
        auto nx = free_blocks.lower_bound(off);
        if (nx != free_blocks.end() && off + size == nx->first) {
            size += nx->second;
            nx = free_blocks.erase(nx);
        }
        if (nx != free_blocks.begin()) {
            auto pv = std::prev(nx);
            if (pv->first + pv->second == off) {
                pv->second += size;
                return;
            }
        }
        free_blocks[off] = size;
    }

    bool contains(const void* p) const {
        const char* c = static_cast<const char*>(p);
        return ok && c >= host_base && c < host_base + capacity;
    }

    bool find(const void* p, ArenaBlock* out) {
        std::lock_guard<std::mutex> g(mu);
        if (!contains(p)) return false;
        size_t off = static_cast<const char*>(p) - host_base;
        auto it = live.upper_bound(off);
        if (it != live.begin()) {
            --it;
            if (off < it->first + it->second.size) {
                if (out) *out = it->second;
                return true;
            }
        }
        if (!pool) return false;
        // a heap object of a captured program: one region up to the pool's high water
        const size_t hw = heap_pool_high_water();
        if (off >= hw) return false;
        if (out) {
            out->offset = 0;
            out->size = hw;
            out->residency = PARALLAX_COHERENT;
        }
        return true;
    }

    // Pool-backed mode: page-locks the pool up to its high-water mark (64 MiB steps, never
    // undone), so kernels can use any pool address. False when registration fails.
    bool lock_pool() {
        std::lock_guard<std::mutex> g(mu);
        const size_t hw = heap_pool_high_water();
        constexpr size_t kStep = 64ull << 20;
        while (pool_locked < hw) {
            const size_t len = capacity - pool_locked < kStep ? capacity - pool_locked : kStep;
            if (cudaHostRegister(host_base + pool_locked, len, cudaHostRegisterDefault) != cudaSuccess) {
                cudaGetLastError();
                // a device that reaches pageable memory itself still sees this range
                if (!pageable) {
                    set_error(PARALLAX_ERR_CUDA,
                              "arena: cannot page-lock the heap pool at offset %zu", pool_locked);
                    return false;
                }
            }
            pool_locked += len;
        }
        return true;
    }

    bool set_residency(const void* p, int mode) {
        std::lock_guard<std::mutex> g(mu);
        if (!contains(p)) return false;
        size_t off = static_cast<const char*>(p) - host_base;
        auto it = live.upper_bound(off);
        if (it == live.begin()) return false;
        --it;
        if (off >= it->first + it->second.size) return false;
        it->second.residency = mode;
        return true;
    }
};

Arena& arena() {
    static Arena* a = new Arena();  // never destroyed: outlives late users at exit
    return *a;
}

}  // namespace

bool arena_contains(const void* p) { return arena().contains(p); }
bool arena_find(const void* p, ArenaBlock* out) { return arena().find(p, out); }
void* arena_dev(const void* p) {
    Arena& a = arena();
    if (!a.contains(p)) return nullptr;
    return reinterpret_cast<void*>(a.dev_base + (static_cast<const char*>(p) - a.host_base));
}
uint64_t arena_host_base() { return reinterpret_cast<uint64_t>(arena().host_base); }
uint64_t arena_dev_base() { return static_cast<uint64_t>(arena().dev_base); }
uint64_t arena_mapped_bytes() {
    Arena& a = arena();
    std::lock_guard<std::mutex> g(a.mu);
    return a.mapped;
}

// The host mirror is page-locked chunk by chunk on first copy, and one copy may not span
// two registrations, so arena copies are split at chunk boundaries (which are also the
// boundaries of the device-side physical allocations).
bool arena_copy_async(void* dst, const void* src, size_t bytes, bool to_device,
                      cudaStream_t s) {
    Arena& a = arena();
    const char* h = static_cast<const char*>(to_device ? src : dst);
    size_t off = static_cast<size_t>(h - a.host_base);
    a.pin_range(off, bytes);
    size_t done = 0;
    while (done < bytes) {
        size_t room = a.chunk - (off + done) % a.chunk;
        size_t len = bytes - done < room ? bytes - done : room;
        cudaError_t e = cudaMemcpyAsync(static_cast<char*>(dst) + done,
                                        static_cast<const char*>(src) + done, len,
                                        to_device ? cudaMemcpyHostToDevice
                                                  : cudaMemcpyDeviceToHost,
                                        s);
        if (!cuda_ok(e, "arena copy")) return false;
        done += len;
    }
    return true;
}

bool arena_zero_copy() {
    Arena& a = arena();
    return a.ok && a.pool;
}
bool arena_host_mapped(const void* p, size_t bytes) {
    Arena& a = arena();
    if (!a.ok || a.pool || !a.host_ptr_ok || !bytes) return false;
    const size_t off = static_cast<size_t>(static_cast<const char*>(p) - a.host_base);
    return a.pinned_range(off, bytes);
}
bool arena_make_accessible() {
    Arena& a = arena();
    return !(a.ok && a.pool) || a.lock_pool();
}

bool arena_sync_coherent(Workspace& ws, bool to_device) {
    Arena& a = arena();
    if (a.ok && a.pool) return a.lock_pool();  // zero-copy: nothing moves
    std::vector<std::pair<size_t, size_t>> ranges;  // [begin, end) offsets
    {
        std::lock_guard<std::mutex> g(a.mu);
        if (!a.ok) return true;
        for (const auto& kv : a.live) {
            const ArenaBlock& b = kv.second;
            if (b.residency != PARALLAX_COHERENT) continue;
            if (!ranges.empty() && ranges.back().second == b.offset) ranges.back().second += b.size;
            else ranges.emplace_back(b.offset, b.offset + b.size);
        }
    }
    for (const auto& r : ranges) {
        char* h = a.host_base + r.first;
        char* d = reinterpret_cast<char*>(a.dev_base) + r.first;
        size_t bytes = r.second - r.first;
        bool ok = to_device ? arena_copy_async(d, h, bytes, true, ws.stream())
                            : arena_copy_async(h, d, bytes, false, ws.stream());
        if (!ok) return false;
    }
    return true;
}

}  // namespace pxb

using namespace pxb;

PXB_EXPORT void* parallax_arena_alloc(size_t size, size_t align) {
    void* p = arena().allocate(size, align ? align : 16);
    static const bool debug = getenv("PARALLAX_DEBUG") != nullptr;
    if (debug)
        fprintf(stderr, "[parallax_arena_alloc] %zu bytes -> %p\n", size, p);
    return p;
}
PXB_EXPORT void parallax_arena_free(void* ptr) {
    settle_deferred_here();  // a held-back transform may read or write this block
    arena().deallocate(ptr);
}
PXB_EXPORT int parallax_arena_contains(const void* ptr) {
    Arena& a = arena();
    if (!a.ok) {
        std::lock_guard<std::mutex> g(a.mu);
        a.init();
    }
    return ptr && a.contains(ptr) ? 1 : 0;
}

PXB_EXPORT void* parallax_umalloc(size_t size, unsigned) { return parallax_arena_alloc(size, 256); }
PXB_EXPORT void parallax_ufree(void* ptr) { parallax_arena_free(ptr); }

PXB_EXPORT int parallax_arena_set_residency(void* ptr, int mode) {
    settle_deferred_here();
    if (mode != PARALLAX_COHERENT && mode != PARALLAX_DEVICE_RESIDENT)
        return PARALLAX_ERR_INVALID_ARGUMENT;
    return arena().set_residency(ptr, mode) ? PARALLAX_OK : PARALLAX_ERR_INVALID_ARGUMENT;
}
PXB_EXPORT int parallax_arena_get_residency(const void* ptr) {
    ArenaBlock b;
    return arena().find(ptr, &b) ? b.residency : -1;
}
PXB_EXPORT void* parallax_arena_device_ptr(const void* host_ptr) { return arena_dev(host_ptr); }
PXB_EXPORT void parallax_arena_bases(uint64_t* host_base, uint64_t* dev_base) {
    Arena& a = arena();
    {
        std::lock_guard<std::mutex> g(a.mu);
        a.init();
    }
    if (host_base) *host_base = reinterpret_cast<uint64_t>(a.host_base);
    if (dev_base) *dev_base = static_cast<uint64_t>(a.dev_base);
}
PXB_EXPORT size_t parallax_arena_capacity(void) {
    Arena& a = arena();
    std::lock_guard<std::mutex> g(a.mu);
    a.init();
    return a.capacity;
}
PXB_EXPORT size_t parallax_arena_used(void) {
    Arena& a = arena();
    std::lock_guard<std::mutex> g(a.mu);
    return a.used;
}
PXB_EXPORT size_t parallax_arena_mapped(void) {
    Arena& a = arena();
    std::lock_guard<std::mutex> g(a.mu);
    return a.mapped;
}

static int arena_copy(const void* ptr, size_t bytes, bool to_device) {
    settle_deferred_here();
    Workspace* ws = workspace();
    if (!ws) return PARALLAX_ERR_NO_DEVICE;
    ArenaBlock b;
    if (!arena().find(ptr, &b)) return PARALLAX_ERR_INVALID_ARGUMENT;
    if (arena_zero_copy()) return PARALLAX_OK;  // one copy, seen by both sides
    size_t off = static_cast<const char*>(ptr) - arena().host_base;
    if (off + bytes > b.offset + b.size) return PARALLAX_ERR_INVALID_ARGUMENT;
    void* dev = arena_dev(ptr);
    bool ok = to_device ? arena_copy_async(dev, ptr, bytes, true, ws->stream())
                        : arena_copy_async(const_cast<void*>(ptr), dev, bytes, false,
                                           ws->stream());
    if (!ok) return PARALLAX_ERR_CUDA;
    return ws->async ? PARALLAX_OK : sync_stream(*ws);
}
PXB_EXPORT int parallax_arena_sync_to_device(const void* ptr, size_t bytes) {
    return arena_copy(ptr, bytes, true);
}
PXB_EXPORT int parallax_arena_sync_to_host(void* ptr, size_t bytes) {
    return arena_copy(ptr, bytes, false);
}
