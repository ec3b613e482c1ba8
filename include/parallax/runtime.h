/*
 * parallax runtime C ABI — B200 (sm_100a) implementation.
 *
 * Every declaration below has the same name, parameter list and return type as the
 * Parallax Runtime ABI that compiler-emitted code and the stdpar funnels link against
 * (reference interface: include/parallax/runtime.h:15-113 and :144-145 in
 * parallax-runtime). Code built against the reference header links against
 * libparallax-runtime.so from this project unchanged.
 *
 * Semantics kept from the reference:
 *  - every call is synchronous from the caller's point of view: results are visible in
 *    host memory when the call returns (reference: src/kernel/cache.cpp:106-392);
 *  - a lookup miss returns NULL and the caller runs its own host loop;
 *  - void calls report errors on stderr and leave outputs unwritten; copy_if returns 0
 *    on failure; argminmax/find/mismatch return `count` on failure.
 * What changes underneath: kernels are sm_100a CUDA (not SPIR-V), the arena is device
 * resident with a pinned host mirror, and calls may come from many host threads.
 * Additive entry points live in parallax/runtime_ext.h.
 */
#ifndef PARALLAX_RUNTIME_H
#define PARALLAX_RUNTIME_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct parallax_runtime* parallax_runtime_t;
typedef struct parallax_kernel* parallax_kernel_t;

/* ---- memory --------------------------------------------------------------------- */

/* Replaces reference runtime.h:16-17 (MemoryManager buffers). Here: an arena block
 * with 256-byte alignment; `flags` is accepted and ignored. */
void* parallax_umalloc(size_t size, unsigned flags);
void parallax_ufree(void* ptr);

/* Replaces reference runtime.h:22-24 (UnifiedArena C accessors,
 * src/memory/unified_allocator.cpp:85-103). The returned pointer is a HOST address in
 * the pinned mirror of a device-resident arena; kernels see the same block at
 * dev_base + (ptr - host_base). Alignment is max(align, 256). NULL when exhausted. */
void* parallax_arena_alloc(size_t size, size_t align);
void parallax_arena_free(void* ptr);
int parallax_arena_contains(const void* ptr);

/* Replaces reference runtime.h:30. Whole-heap capture is not built; always 0. */
int parallax_heap_contains(const void* ptr);

/* ---- kernel handles and element-wise launches ------------------------------------ */

/* Replaces reference runtime.h:33. `image` is a CUDA cubin or fatbin for sm_100a
 * (`words` 32-bit words). A SPIR-V image is rejected (NULL). */
parallax_kernel_t parallax_kernel_load(const unsigned int* spirv, size_t words);

/* Replaces reference runtime.h:34. Variadic: (void* buffer, size_t count,
 * size_t elem_size), as read in reference src/kernel/cache.cpp:114-120. */
void parallax_kernel_launch(parallax_kernel_t kernel, ...);

/* Replaces reference runtime.h:35. Variadic: (void* in, void* out, size_t count,
 * size_t elem_size), as read in reference src/kernel/cache.cpp:155-162. */
void parallax_kernel_launch_transform(parallax_kernel_t kernel, ...);

/* Replaces reference runtime.h:37-39. */
void parallax_kernel_launch_transform2(parallax_kernel_t kernel, void* in_buffer,
                                       void* out_buffer, size_t count,
                                       size_t in_elem_size, size_t out_elem_size);

/* Replaces reference runtime.h:43-46. The capture bytes are copied at call time. */
void parallax_kernel_launch_transform2_captures(parallax_kernel_t kernel, void* in_buffer,
                                                void* out_buffer, size_t count,
                                                size_t in_elem_size, size_t out_elem_size,
                                                void* captures, size_t capture_size);

/* ---- primitives ------------------------------------------------------------------ */

/* Replaces reference runtime.h:52-53. Writes elem_size bytes of the reduction of
 * data[0..count) (without any init) to `result`. The operation (sum, max, ...) and
 * the element type are properties of the handle. */
void parallax_reduce(parallax_kernel_t kernel, void* data, size_t count,
                     size_t elem_size, void* result);

/* Replaces reference runtime.h:59-60. Index of the first minimum (want_max == 0) or
 * maximum; with want_last the last one. 0 for count <= 1, `count` on error. */
size_t parallax_argminmax(parallax_kernel_t kernel, void* data, size_t count,
                          size_t elem_size, int is_float, int want_max, int want_last);

/* Replaces reference runtime.h:64-65. First index whose element satisfies the handle's
 * predicate (negated when negate != 0), or `count`. `value`, when non-NULL, replaces
 * the predicate's operand (find(value) semantics). */
size_t parallax_find(parallax_kernel_t kernel, void* data, size_t count,
                     size_t elem_size, int negate, const void* value);

/* Replaces reference runtime.h:68. First index where a[i] != b[i], or `count`. */
size_t parallax_mismatch(parallax_kernel_t kernel, void* a, void* b, size_t count,
                         size_t elem_size);

/* Replaces reference runtime.h:72-73. In-place inclusive '+' scan. add_kernel must be
 * non-NULL (the single-pass scan does not need it). */
void parallax_scan(parallax_kernel_t scan_kernel, parallax_kernel_t add_kernel,
                   void* data, size_t count, size_t elem_size);

/* Replaces reference runtime.h:78-80. output[i] = init + sum(input[0..i)); `init`
 * points at elem_size bytes. `input` is read only (the reference may clobber it). */
void parallax_exclusive_scan(parallax_kernel_t scan_kernel, parallax_kernel_t add_kernel,
                             parallax_kernel_t shift_kernel, void* input, void* output,
                             size_t count, size_t elem_size, const void* init);

/* Replaces reference runtime.h:85. In-place ascending sort. Any count is accepted (the
 * reference requires a power of two). Floating-point keys are ordered by the IEEE total
 * order, so -0.0 sorts before +0.0; this is a valid result for operator<. */
void parallax_sort(parallax_kernel_t kernel, void* data, size_t count, size_t elem_size);

/* Replaces reference runtime.h:91-94. Stable compaction. The flags handle selects the
 * predicate (copy_if / remove_if) or adjacent-difference (unique); a partition scatter
 * handle turns it into a stable partition that writes all `count` elements and
 * returns the number of elements for which the predicate holds. */
size_t parallax_copy_if(parallax_kernel_t flags_kernel, parallax_kernel_t scan_kernel,
                        parallax_kernel_t add_kernel, parallax_kernel_t scatter_kernel,
                        void* input, void* output, size_t count, size_t elem_size,
                        int elem_is_float);

/* ---- registry -------------------------------------------------------------------- */

/* Replaces reference runtime.h:102-103 (src/kernel/cache.cpp:83-104). Registration only
 * records the pointer (safe at static-init time). Lookup resolves a registered sm_100a
 * image lazily, or a built-in sm_100a kernel when the key names a primitive funnel
 * instantiation (device_reduce<T>, device_scan<T>:scan, device_sort<T>, ...). */
void parallax_kernel_register(const char* key, const unsigned int* spirv, size_t words);
parallax_kernel_t parallax_kernel_lookup(const char* key);

/* Replaces reference runtime.h:106-113. */
void parallax_kernel_launch_with_captures(
    parallax_kernel_t kernel,
    void* buffer,
    size_t count,
    void* captures,
    size_t capture_size,
    size_t elem_size
);

#ifdef __cplusplus
}
#endif

#ifdef __cplusplus
/* Same template as reference runtime.h:129-139: the funnels offload only contiguous
 * iterator ranges. */
#include <iterator>
#include <type_traits>
namespace parallax {
#if __cplusplus >= 202002L
template <class It>
inline constexpr bool is_contiguous_iterator_v =
    std::contiguous_iterator<std::remove_cvref_t<It>>;
#else
template <class It>
inline constexpr bool is_contiguous_iterator_v =
    std::is_pointer_v<std::remove_reference_t<It>>;
#endif
}  // namespace parallax
#endif /* __cplusplus */

#endif /* PARALLAX_RUNTIME_H */

/* Replaces reference runtime.h:144-145. Declared outside the include guard and outside
 * extern "C" in the reference, so it is a C++-linkage (mangled) symbol; kept that way
 * for link compatibility. Pins the host range for fast staging; returns true. */
#ifdef __cplusplus
bool parallax_register_buffer(void* ptr, size_t size);
#endif
