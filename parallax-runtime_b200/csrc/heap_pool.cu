// Process-wide heap pool: the substrate of whole-heap capture.
//
// Replaces the reference's heap pool (src/memory/heap_pool.cpp:90-195, API
// include/parallax/heap_pool.hpp:20-60; same names, argument meanings and environment
// variables, so a program or capture shim written against the reference links unchanged).
// One anonymous MAP_NORESERVE reservation (PARALLAX_HEAP_POOL MiB, default 8 GiB, 2 MiB
// aligned) holds every block; pages are backed only when touched. When the pool is live
// before the runtime first uses its arena, the arena adopts the reservation as its host
// mirror (arena.cu): heap pointers are then arena pointers, operands move between the
// pool and HBM exactly like arena blocks, and stored heap pointers relocate with the
// arena formula dev_base + (p - host_base).
//
// The allocator allocates nothing itself (no malloc, no C++ containers; mmap and static
// storage only), so a malloc / operator new interposer may call it at any time, before
// main and from inside the CUDA runtime. Design (not the reference's): boundary tags and
// segregated free lists.
//   * a block starts with a 16-byte header {size | flags, unused}; its payload starts at
//     header + 16 and is 16-byte aligned; sizes are multiples of 16, at least 48;
//   * flags: bit 0 the block is in use, bit 1 the block before it is in use; a free block
//     repeats its size in its last 8 bytes (the footer), so a freed neighbour can find it;
//   * free blocks sit in one of 64 doubly linked lists by floor(log2(size)); allocation
//     takes the first fitting block of the smallest list that can hold it, splitting off
//     the remainder; never-used space is one "top" region at the end, carved on demand;
//   * freeing coalesces with free neighbours and returns space that ends at the top to it.
// One spin lock (an atomic flag) guards the lists. PARALLAX_HEAP_CHECK=1 walks and checks
// every block after each operation (tests).
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <sys/mman.h>

#include <atomic>

#include "runtime.hpp"

#define PXP_EXPORT extern "C" __attribute__((visibility("default")))

namespace pxb {
namespace {

constexpr size_t kHdr = 16;
constexpr size_t kMinBlock = 48;
constexpr size_t kBins = 64;
constexpr uint64_t kUsed = 1, kPrevUsed = 2, kFlags = 15;

struct FreeLinks {
    char* next;
    char* prev;
};

std::atomic_flag g_lock = ATOMIC_FLAG_INIT;
std::atomic<char*> g_base{nullptr};
std::atomic<size_t> g_reservation{0};
std::atomic<size_t> g_high{0};   // bytes ever carved from the top
bool g_tried = false;
bool g_check = false;
char* g_top = nullptr;            // first byte of the never-used region
char* g_end = nullptr;
char* g_bins[kBins];

struct Guard {
    Guard() {
        while (g_lock.test_and_set(std::memory_order_acquire)) __builtin_ia32_pause();
    }
    ~Guard() { g_lock.clear(std::memory_order_release); }
};

inline size_t round_up(size_t v, size_t a) { return (v + a - 1) / a * a; }
inline uint64_t& head(char* b) { return *reinterpret_cast<uint64_t*>(b); }
inline size_t bsize(char* b) { return (size_t)(head(b) & ~kFlags); }
inline bool used(char* b) { return (head(b) & kUsed) != 0; }
inline bool prev_used(char* b) { return (head(b) & kPrevUsed) != 0; }
inline FreeLinks* links(char* b) { return reinterpret_cast<FreeLinks*>(b + kHdr); }
inline void set_footer(char* b) { *reinterpret_cast<uint64_t*>(b + bsize(b) - 8) = bsize(b); }
inline char* block_of(const void* payload) { return (char*)payload - kHdr; }

int bin_of(size_t size) { return 63 - __builtin_clzll((unsigned long long)size); }

void bin_remove(char* b) {
    FreeLinks* l = links(b);
    if (l->prev) links(l->prev)->next = l->next;
    else g_bins[bin_of(bsize(b))] = l->next;
    if (l->next) links(l->next)->prev = l->prev;
}
void bin_insert(char* b) {
    const int i = bin_of(bsize(b));
    FreeLinks* l = links(b);
    l->prev = nullptr;
    l->next = g_bins[i];
    if (g_bins[i]) links(g_bins[i])->prev = b;
    g_bins[i] = b;
}

// The block after b (or g_top); marks its "previous in use" flag.
void set_next_prev_used(char* b, bool in_use) {
    char* n = b + bsize(b);
    if (n >= g_top) return;
    if (in_use) head(n) |= kPrevUsed;
    else head(n) &= ~kPrevUsed;
}

bool init_locked() {
    if (g_tried) return g_base.load(std::memory_order_relaxed) != nullptr;
    g_tried = true;
    if (const char* e = getenv("PARALLAX_HEAP_CHECK")) g_check = e[0] && e[0] != '0';
    size_t res = 8ull << 30;
    if (const char* e = getenv("PARALLAX_HEAP_POOL")) {
        const long long v = atoll(e);  // MiB
        if (v > 0) res = (size_t)v << 20;
    }
    constexpr size_t kAlignment = 2ull << 20;  // arena chunks and page-lock ranges align to it
    res = round_up(res, kAlignment);
    void* p = mmap(nullptr, res + kAlignment, PROT_READ | PROT_WRITE,
                   MAP_PRIVATE | MAP_ANONYMOUS | MAP_NORESERVE, -1, 0);
    if (p == MAP_FAILED) return false;
    char* base = (char*)round_up((uintptr_t)p, kAlignment);
    for (size_t i = 0; i < kBins; ++i) g_bins[i] = nullptr;
    g_top = base;
    g_end = base + res;
    g_reservation.store(res, std::memory_order_relaxed);
    g_base.store(base, std::memory_order_release);
    return true;
}

// Carves `size` bytes from the top; nullptr when the reservation is exhausted.
char* from_top(size_t size, bool prev_in_use) {
    if ((size_t)(g_end - g_top) < size) return nullptr;
    char* b = g_top;
    g_top += size;
    g_high.store((size_t)(g_top - g_base.load(std::memory_order_relaxed)),
                 std::memory_order_relaxed);
    head(b) = size | kUsed | (prev_in_use ? kPrevUsed : 0);
    return b;
}

void free_locked(char* b);

// Splits used block b to `size` bytes when the rest can be a block of its own; the rest is
// freed (merged with a free successor, or given back to the top).
void trim(char* b, size_t size) {
    const size_t have = bsize(b);
    if (have - size < kMinBlock) return;
    char* r = b + size;
    head(b) = size | (head(b) & kFlags);
    head(r) = (have - size) | kUsed | kPrevUsed;
    free_locked(r);
}

char* alloc_locked(size_t n, size_t align) {
    if (!init_locked()) return nullptr;
    if (align < 16) align = 16;
    align = (size_t)1 << (64 - __builtin_clzll((unsigned long long)(align - 1)));  // power of 2
    const size_t need = round_up(n + kHdr, 16) < kMinBlock ? kMinBlock : round_up(n + kHdr, 16);
    // over-allocate for alignments above 16: room to split off an aligned front
    const size_t want = align > 16 ? need + align + kMinBlock : need;
    char* b = nullptr;
    for (int i = bin_of(want); i < (int)kBins && !b; ++i)
        for (char* c = g_bins[i]; c; c = links(c)->next)
            if (bsize(c) >= want) {
                b = c;
                break;
            }
    if (b) {
        bin_remove(b);
        head(b) |= kUsed;
        set_next_prev_used(b, true);
    } else {
        // free blocks never touch the top (they merge into it), so the block below the
        // top is always in use
        b = from_top(want, true);
        if (!b) return nullptr;
    }
    if (align > 16) {
        // first payload address >= b + kHdr that is aligned, leaving a front gap of zero or
        // at least kMinBlock (a block of its own)
        uintptr_t pay = round_up((uintptr_t)(b + kHdr), align);
        if (pay - kHdr != (uintptr_t)b && pay - kHdr - (uintptr_t)b < kMinBlock)
            pay = round_up((uintptr_t)(b + kHdr + kMinBlock), align);
        char* a = (char*)(pay - kHdr);
        if (a != b) {  // free the front part
            const size_t front = (size_t)(a - b), total = bsize(b);
            const uint64_t pf = head(b) & kPrevUsed;
            head(b) = front | pf;
            set_footer(b);
            head(a) = (total - front) | kUsed;  // previous (the front) is free
            bin_insert(b);
            b = a;
        }
    }
    trim(b, need);
    return b;
}

void free_locked(char* b) {
    char* base = g_base.load(std::memory_order_relaxed);
    size_t size = bsize(b);
    // coalesce with the following free block
    char* n = b + size;
    if (n < g_top && !used(n)) {
        bin_remove(n);
        size += bsize(n);
    }
    // coalesce with the preceding free block
    uint64_t keep = kPrevUsed;
    if (!prev_used(b) && b > base) {
        const size_t ps = (size_t)*reinterpret_cast<uint64_t*>(b - 8);
        char* p = b - ps;
        bin_remove(p);
        size += ps;
        b = p;
        keep = head(p) & kPrevUsed;
    } else {
        keep = head(b) & kPrevUsed;
    }
    if (b + size == g_top) {  // back to the top
        g_top = b;
        return;
    }
    head(b) = size | keep;
    set_footer(b);
    set_next_prev_used(b, false);
    bin_insert(b);
}

int check_locked() {
    char* base = g_base.load(std::memory_order_relaxed);
    if (!base) return 1;
    bool prev_in_use = true;
    size_t free_blocks = 0;
    for (char* b = base; b < g_top;) {
        const size_t s = bsize(b);
        if (s < kMinBlock || s % 16 || b + s > g_top) return 0;
        if (prev_used(b) != prev_in_use) return 0;
        if (!used(b)) {
            if (!prev_in_use) return 0;  // two free neighbours were not coalesced
            if (*reinterpret_cast<uint64_t*>(b + s - 8) != s) return 0;
            ++free_blocks;
        }
        prev_in_use = used(b);
        b += s;
    }
    size_t listed = 0;
    for (size_t i = 0; i < kBins; ++i)
        for (char* c = g_bins[i]; c; c = links(c)->next) {
            if (used(c) || bin_of(bsize(c)) != (int)i) return 0;
            if (++listed > free_blocks) return 0;
        }
    return listed == free_blocks;
}

void maybe_check() {
    if (g_check && !check_locked()) abort();
}

}  // namespace

void* heap_pool_base() { return g_base.load(std::memory_order_acquire); }
size_t heap_pool_reservation() { return g_reservation.load(std::memory_order_acquire); }
size_t heap_pool_high_water() { return g_high.load(std::memory_order_relaxed); }

}  // namespace pxb

using namespace pxb;

PXP_EXPORT int px_pool_init(void) {
    Guard g;
    return init_locked() ? 1 : 0;
}

PXP_EXPORT void* px_pool_alloc(size_t size, size_t align) {
    Guard g;
    char* b = alloc_locked(size, align);
    maybe_check();
    return b ? b + kHdr : nullptr;
}

PXP_EXPORT int px_pool_contains(const void* ptr) {
    const char* base = g_base.load(std::memory_order_acquire);
    if (!base || !ptr) return 0;
    const char* p = static_cast<const char*>(ptr);
    return p >= base && p < base + g_reservation.load(std::memory_order_relaxed) ? 1 : 0;
}

PXP_EXPORT void px_pool_free(void* ptr) {
    if (!ptr) return;
    Guard g;
    free_locked(block_of(ptr));
    maybe_check();
}

PXP_EXPORT size_t px_pool_usable_size(const void* ptr) {
    if (!ptr) return 0;
    return bsize(block_of(ptr)) - kHdr;
}

PXP_EXPORT void* px_pool_realloc(void* ptr, size_t new_size) {
    if (!ptr) return px_pool_alloc(new_size, 16);
    if (new_size == 0) {
        px_pool_free(ptr);
        return nullptr;
    }
    {
        Guard g;
        char* b = block_of(ptr);
        const size_t need = round_up(new_size + kHdr, 16) < kMinBlock ? kMinBlock
                                                                      : round_up(new_size + kHdr, 16);
        if (need <= bsize(b)) {  // shrink in place
            trim(b, need);
            maybe_check();
            return ptr;
        }
        char* n = b + bsize(b);
        if (n < g_top && !used(n) && bsize(b) + bsize(n) >= need) {  // grow into the next block
            bin_remove(n);
            head(b) = (bsize(b) + bsize(n)) | (head(b) & kFlags);
            set_next_prev_used(b, true);
            trim(b, need);
            maybe_check();
            return ptr;
        }
        if (n == g_top && (size_t)(g_end - g_top) >= need - bsize(b)) {  // grow into the top
            g_top += need - bsize(b);
            g_high.store((size_t)(g_top - g_base.load(std::memory_order_relaxed)),
                         std::memory_order_relaxed);
            head(b) = need | (head(b) & kFlags);
            maybe_check();
            return ptr;
        }
    }
    void* q = px_pool_alloc(new_size, 16);
    if (!q) return nullptr;
    memcpy(q, ptr, px_pool_usable_size(ptr));
    px_pool_free(ptr);
    return q;
}

PXP_EXPORT void* px_pool_base(void) { return g_base.load(std::memory_order_acquire); }
PXP_EXPORT size_t px_pool_reservation(void) { return g_reservation.load(std::memory_order_acquire); }
PXP_EXPORT size_t px_pool_high_water(void) { return g_high.load(std::memory_order_relaxed); }

PXP_EXPORT int px_pool_check(void) {
    Guard g;
    return check_locked();
}

// Whole-heap capture membership (runtime.h): 1 iff ptr lies in the pool's reservation.
PXP_EXPORT int parallax_heap_contains(const void* ptr) { return px_pool_contains(ptr); }
