// Whole-heap capture: links into a program (lib/libparallax-heap.a) and routes every heap
// allocation the program makes into the runtime's heap pool (csrc/heap_pool.cu).
//
// Replaces the reference's capture shim (src/memory/heap_capture.cpp:47-126, the
// parallax-heap static library its compiler wrapper links): strong definitions of the
// malloc family and of every operator new / delete override the C library's and the C++
// library's, so std::vector storage and everything else on the heap lands in the pool.
// When the runtime's arena starts while the pool is live, the arena adopts the pool as its
// host mirror: heap pointers handed to the ABI are then arena pointers (moved to and from
// HBM by range, no staging copy), and pointers stored inside heap objects relocate with
// dev_base + (p - host_base) in kernels.
//
// Pointers that did not come from the pool (allocated before it existed, or when it is
// exhausted) go back to the C library's own allocator through its __libc_* entry points;
// calling the public names here would call these definitions again. Linux / glibc only.
#include <stddef.h>
#include <string.h>

#include <new>

#include "parallax/heap_pool.h"

extern "C" {
void* __libc_malloc(size_t);
void* __libc_calloc(size_t, size_t);
void* __libc_realloc(void*, size_t);
void* __libc_memalign(size_t, size_t);
void __libc_free(void*);
}

namespace {

void* take(size_t n, size_t align) {
    void* p = px_pool_alloc(n ? n : 1, align);
    return p ? p : (align <= 16 ? __libc_malloc(n ? n : 1) : __libc_memalign(align, n ? n : 1));
}

void give_back(void* p) {
    if (!p) return;
    if (px_pool_contains(p)) px_pool_free(p);
    else __libc_free(p);
}

void* take_or_throw(size_t n, size_t align) {
    void* p = take(n, align);
    if (!p) throw std::bad_alloc();
    return p;
}

}  // namespace

extern "C" {

void* malloc(size_t n) { return take(n, 16); }
void free(void* p) { give_back(p); }
void* calloc(size_t count, size_t size) {
    if (size && count > (size_t)-1 / size) return nullptr;
    const size_t n = count * size;
    void* p = px_pool_alloc(n ? n : 1, 16);
    if (!p) return __libc_calloc(count ? count : 1, size ? size : 1);
    memset(p, 0, n);  // a reused pool block is not zero
    return p;
}
void* realloc(void* p, size_t n) {
    if (!p) return take(n, 16);
    if (px_pool_contains(p)) {
        if (n == 0) {
            px_pool_free(p);
            return nullptr;
        }
        return px_pool_realloc(p, n);
    }
    return __libc_realloc(p, n);
}
void* aligned_alloc(size_t align, size_t n) { return take(n, align); }
void* memalign(size_t align, size_t n) { return take(n, align); }
int posix_memalign(void** out, size_t align, size_t n) {
    if (align < sizeof(void*) || (align & (align - 1))) return 22;  // EINVAL
    void* p = take(n, align);
    if (!p) return 12;  // ENOMEM
    *out = p;
    return 0;
}
void* valloc(size_t n) { return take(n, 4096); }
void* pvalloc(size_t n) { return take((n + 4095) / 4096 * 4096, 4096); }
size_t malloc_usable_size(void* p) {
    if (!p) return 0;
    if (px_pool_contains(p)) return px_pool_usable_size(p);
    return 0;  // a C-library block: its size is not known here
}

}  // extern "C"

void* operator new(size_t n) { return take_or_throw(n, 16); }
void* operator new[](size_t n) { return take_or_throw(n, 16); }
void* operator new(size_t n, std::align_val_t a) { return take_or_throw(n, (size_t)a); }
void* operator new[](size_t n, std::align_val_t a) { return take_or_throw(n, (size_t)a); }
void* operator new(size_t n, const std::nothrow_t&) noexcept { return take(n, 16); }
void* operator new[](size_t n, const std::nothrow_t&) noexcept { return take(n, 16); }
void* operator new(size_t n, std::align_val_t a, const std::nothrow_t&) noexcept {
    return take(n, (size_t)a);
}
void* operator new[](size_t n, std::align_val_t a, const std::nothrow_t&) noexcept {
    return take(n, (size_t)a);
}
void operator delete(void* p) noexcept { give_back(p); }
void operator delete[](void* p) noexcept { give_back(p); }
void operator delete(void* p, size_t) noexcept { give_back(p); }
void operator delete[](void* p, size_t) noexcept { give_back(p); }
void operator delete(void* p, std::align_val_t) noexcept { give_back(p); }
void operator delete[](void* p, std::align_val_t) noexcept { give_back(p); }
void operator delete(void* p, size_t, std::align_val_t) noexcept { give_back(p); }
void operator delete[](void* p, size_t, std::align_val_t) noexcept { give_back(p); }
void operator delete(void* p, const std::nothrow_t&) noexcept { give_back(p); }
void operator delete[](void* p, const std::nothrow_t&) noexcept { give_back(p); }
