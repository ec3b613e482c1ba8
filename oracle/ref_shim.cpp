// The reference's own CPU path, compiled from its unmodified header. TEST
// INFRASTRUCTURE ONLY (oracle pin and timed CPU baseline); never linked into the runtime.
//
// include/parallax/stdpar.hpp (parallax-runtime) offloads every algorithm through
// parallax_kernel_lookup() and runs its ISO host loop when the lookup misses
// (stdpar.hpp:46-394). This file is linked with an ABI whose lookup always misses
// (abi_stub.cpp), so each parallax::* call below executes exactly the reference's host
// fallback:
//   reduce stdpar.hpp:146-148, inclusive_scan :209-210, exclusive_scan :237-238,
//   sort :178, copy_if :319-321, remove_if :343-345, partition :369-370, unique :392-393.
// Built by oracle/Makefile against -I <reference>/include into oracle/_ref/.
#include <parallax/stdpar.hpp>

#include <stdint.h>

#define RX extern "C" __attribute__((visibility("default")))

namespace {
struct Mod3 { bool operator()(int32_t x) const { return x % 3 == 0; } };
struct Neg { bool operator()(int32_t x) const { return x < 0; } };
struct GtHalfF { bool operator()(float x) const { return x > 0.5f; } };
struct GtHalfD { bool operator()(double x) const { return x > 0.5; } };
struct GtHalfI { bool operator()(int32_t x) const { return x > 0; } };
}  // namespace

// ---- exported entry points (element types of the benchmark configurations) ---------------
#define REF_FOLD(sfx, T)                                                                    \
    RX T ref_reduce_##sfx(const T* x, size_t n) {                                            \
        return parallax::reduce(parallax::par, x, x + n, T{});                               \
    }                                                                                        \
    RX void ref_inclusive_scan_##sfx(const T* x, T* out, size_t n) {                         \
        parallax::inclusive_scan(parallax::par, x, x + n, out);                              \
    }                                                                                        \
    RX void ref_exclusive_scan_##sfx(const T* x, T* out, size_t n, T init) {                 \
        parallax::exclusive_scan(parallax::par, x, x + n, out, init);                        \
    }                                                                                        \
    RX void ref_sort_##sfx(T* x, size_t n) { parallax::sort(parallax::par, x, x + n); }      \
    RX size_t ref_unique_##sfx(T* x, size_t n) {                                             \
        return (size_t)(parallax::unique(parallax::par, x, x + n) - x);                      \
    }
REF_FOLD(f32, float)
REF_FOLD(f64, double)
REF_FOLD(i32, int32_t)
REF_FOLD(i64, int64_t)
REF_FOLD(u32, uint32_t)
REF_FOLD(u64, uint64_t)

RX size_t ref_copy_if_mod3_i32(const int32_t* x, int32_t* out, size_t n) {
    return (size_t)(parallax::copy_if(parallax::par, x, x + n, out, Mod3{}) - out);
}
RX size_t ref_remove_if_mod3_i32(int32_t* x, size_t n) {
    return (size_t)(parallax::remove_if(parallax::par, x, x + n, Mod3{}) - x);
}
RX size_t ref_partition_neg_i32(int32_t* x, size_t n) {
    return (size_t)(parallax::partition(parallax::par, x, x + n, Neg{}) - x);
}
RX size_t ref_copy_if_gthalf_f32(const float* x, float* out, size_t n) {
    return (size_t)(parallax::copy_if(parallax::par, x, x + n, out, GtHalfF{}) - out);
}
RX size_t ref_copy_if_gthalf_f64(const double* x, double* out, size_t n) {
    return (size_t)(parallax::copy_if(parallax::par, x, x + n, out, GtHalfD{}) - out);
}
RX size_t ref_copy_if_gt0_i32(const int32_t* x, int32_t* out, size_t n) {
    return (size_t)(parallax::copy_if(parallax::par, x, x + n, out, GtHalfI{}) - out);
}
