/*
 * Heap pool of whole-heap capture, exported by libparallax-runtime.so.
 *
 * Same functions, argument meanings and environment variables as the reference's
 * include/parallax/heap_pool.hpp:20-60 (src/memory/heap_pool.cpp), so a capture shim or a
 * program written against the reference links unchanged. One process-wide MAP_NORESERVE
 * reservation (PARALLAX_HEAP_POOL MiB, default 8192) that allocates only with mmap and
 * static storage, so a malloc / operator new replacement (lib/libparallax-heap.a) can call
 * it before main. When the pool is live before the runtime's arena starts, the arena
 * adopts the reservation as its host mirror: every pool pointer is an arena pointer (see
 * parallax_arena_contains) and is relocated in kernels like one.
 */
#ifndef PARALLAX_HEAP_POOL_H
#define PARALLAX_HEAP_POOL_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* `size` bytes aligned to at least `align` (rounded up to a power of two >= 16); NULL when
 * the reservation is exhausted. Thread-safe. */
void* px_pool_alloc(size_t size, size_t align);
/* Frees a pointer from px_pool_alloc / px_pool_realloc (callers check px_pool_contains
 * first). Thread-safe. */
void px_pool_free(void* ptr);
/* Keeps min(old, new) bytes; NULL ptr allocates, size 0 frees and returns NULL. */
void* px_pool_realloc(void* ptr, size_t new_size);
/* Bytes usable at a pool pointer (>= the size asked for). */
size_t px_pool_usable_size(const void* ptr);
/* 1 iff ptr lies inside the reservation; 0 when the pool was never initialized. */
int px_pool_contains(const void* ptr);
/* Base of the reservation (2 MiB aligned) and its size; NULL / 0 before initialization. */
void* px_pool_base(void);
size_t px_pool_reservation(void);
/* Highest offset ever handed out. */
size_t px_pool_high_water(void);
/* Initializes the pool now (idempotent); 1 on success, 0 when the reservation failed. */
int px_pool_init(void);
/* Walks every block and checks the allocator's invariants; 1 when they hold
 * (PARALLAX_HEAP_CHECK=1 runs it after every operation). */
int px_pool_check(void);

#ifdef __cplusplus
}
#endif

#endif /* PARALLAX_HEAP_POOL_H */
