// The primitives under std::execution::par, as the host C++ library provides them.
// TEST / BENCHMARK INFRASTRUCTURE ONLY: bench.py times these beside the reference's own
// host fallbacks (libparallax_ref.so) as the "std::execution::par on the host's cores"
// baseline; nothing here is linked into the runtime.
//
// libstdc++ runs the parallel policies on oneTBB when it is installed and otherwise on its
// serial backend; pstl_backend() names the one this build got, and pstl_threads() the host's
// hardware concurrency.
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <execution>
#include <numeric>
#include <thread>

#define PX extern "C" __attribute__((visibility("default")))

PX const char* pstl_backend(void) {
#if defined(_PSTL_PAR_BACKEND_TBB)
    return "libstdc++ PSTL, oneTBB backend";
#elif defined(_PSTL_PAR_BACKEND_OPENMP)
    return "libstdc++ PSTL, OpenMP backend";
#elif defined(_PSTL_PAR_BACKEND_SERIAL)
    return "libstdc++ PSTL, serial backend (oneTBB not installed)";
#else
    return "libstdc++ PSTL, backend unknown";
#endif
}

PX unsigned pstl_threads(void) { return std::thread::hardware_concurrency(); }

#define PSTL_FOLD(sfx, T)                                                                    \
    PX T pstl_reduce_##sfx(const T* x, size_t n) {                                            \
        return std::reduce(std::execution::par, x, x + n, T{});                               \
    }                                                                                         \
    PX void pstl_inclusive_scan_##sfx(const T* x, T* out, size_t n) {                         \
        std::inclusive_scan(std::execution::par, x, x + n, out);                              \
    }                                                                                         \
    PX void pstl_exclusive_scan_##sfx(const T* x, T* out, size_t n, T init) {                 \
        std::exclusive_scan(std::execution::par, x, x + n, out, init);                        \
    }                                                                                         \
    PX void pstl_sort_##sfx(T* x, size_t n) { std::sort(std::execution::par, x, x + n); }
PSTL_FOLD(f32, float)
PSTL_FOLD(f64, double)
PSTL_FOLD(i32, int32_t)
PSTL_FOLD(i64, int64_t)
PSTL_FOLD(u32, uint32_t)

PX size_t pstl_copy_if_mod3_i32(const int32_t* x, int32_t* out, size_t n) {
    return (size_t)(std::copy_if(std::execution::par, x, x + n, out,
                                 [](int32_t v) { return v % 3 == 0; }) - out);
}
PX size_t pstl_partition_neg_i32(int32_t* x, size_t n) {
    return (size_t)(std::stable_partition(std::execution::par, x, x + n,
                                          [](int32_t v) { return v < 0; }) - x);
}
PX size_t pstl_unique_i32(int32_t* x, size_t n) {
    return (size_t)(std::unique(std::execution::par, x, x + n) - x);
}
