// An ABI whose kernel lookup always misses. TEST INFRASTRUCTURE ONLY.
//
// include/parallax/stdpar.hpp (parallax-runtime) offloads every algorithm through
// parallax_kernel_lookup() and runs its ISO host loop when the lookup misses
// (stdpar.hpp:46-394). Linked into the reference's compiled CPU path (ref_shim.cpp) and
// into the host build of stdpar_driver.cpp, it makes every parallax::* call execute
// exactly the reference's host fallback. The symbols are hidden so a shared library built
// with them never interposes the runtime's exports.
#include <parallax/runtime.h>

#include <stdio.h>
#include <stdlib.h>

#define HID __attribute__((visibility("hidden")))

// ---- stub ABI: every lookup misses -------------------------------------------------------
extern "C" {
HID parallax_kernel_t parallax_kernel_lookup(const char*) { return nullptr; }
HID void parallax_kernel_register(const char*, const unsigned int*, size_t) {}
HID int parallax_arena_contains(const void*) { return 0; }
HID int parallax_heap_contains(const void*) { return 0; }
HID void* parallax_arena_alloc(size_t, size_t) { return nullptr; }
HID void parallax_arena_free(void*) {}
static void unreachable(const char* f) {
    fprintf(stderr, "ref_shim: %s reached (lookups miss, so this is a bug)\n", f);
    abort();
}
HID void parallax_kernel_launch(parallax_kernel_t, ...) { unreachable("launch"); }
HID void parallax_kernel_launch_with_captures(parallax_kernel_t, void*, size_t, void*, size_t,
                                              size_t) { unreachable("launch_with_captures"); }
HID void parallax_kernel_launch_transform2(parallax_kernel_t, void*, void*, size_t, size_t,
                                           size_t) { unreachable("transform2"); }
HID void parallax_kernel_launch_transform2_captures(parallax_kernel_t, void*, void*, size_t,
                                                    size_t, size_t, void*, size_t) {
    unreachable("transform2_captures");
}
HID void parallax_reduce(parallax_kernel_t, void*, size_t, size_t, void*) { unreachable("reduce"); }
HID void parallax_scan(parallax_kernel_t, parallax_kernel_t, void*, size_t, size_t) {
    unreachable("scan");
}
HID void parallax_exclusive_scan(parallax_kernel_t, parallax_kernel_t, parallax_kernel_t, void*,
                                 void*, size_t, size_t, const void*) {
    unreachable("exclusive_scan");
}
HID void parallax_sort(parallax_kernel_t, void*, size_t, size_t) { unreachable("sort"); }
HID size_t parallax_copy_if(parallax_kernel_t, parallax_kernel_t, parallax_kernel_t,
                            parallax_kernel_t, void*, void*, size_t, size_t, int) {
    unreachable("copy_if");
    return 0;
}
}
