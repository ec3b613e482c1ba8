// Links the whole-heap capture shim (lib/libparallax-heap.a) and the runtime: every heap
// allocation of this program must come from the runtime's heap pool, and the pool's
// invariants must hold after a mixed workload. Built and run by tests/test_heap_pool.py.
#include <parallax/heap_pool.h>
#include <parallax/runtime.h>

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <map>
#include <memory>
#include <string>
#include <vector>

#define CHECK(c)                                                  \
    do {                                                          \
        if (!(c)) {                                               \
            fprintf(stderr, "check failed: %s (line %d)\n", #c, __LINE__); \
            return 1;                                             \
        }                                                         \
    } while (0)

struct alignas(256) Wide {
    unsigned char b[256];
};

int main() {
    std::vector<int> v(1 << 20, 7);
    CHECK(parallax_heap_contains(v.data()) == 1);
    CHECK(px_pool_contains(v.data()) == 1);
    std::string s(100000, 'x');
    CHECK(parallax_heap_contains(s.data()) == 1);
    std::map<int, std::string> m;
    for (int i = 0; i < 10000; ++i) m[i] = std::to_string(i * 7);
    CHECK(parallax_heap_contains(&m.begin()->second) == 1);
    auto w = std::make_unique<Wide>();
    CHECK(parallax_heap_contains(w.get()) == 1 && reinterpret_cast<uintptr_t>(w.get()) % 256 == 0);
    int* c = static_cast<int*>(calloc(5000, sizeof(int)));
    CHECK(c && parallax_heap_contains(c) == 1);
    for (int i = 0; i < 5000; ++i) CHECK(c[i] == 0);
    for (int i = 0; i < 5000; ++i) c[i] = i;
    c = static_cast<int*>(realloc(c, 200000 * sizeof(int)));
    CHECK(c && parallax_heap_contains(c) == 1);
    for (int i = 0; i < 5000; ++i) CHECK(c[i] == i);
    free(c);
    void* a = nullptr;
    CHECK(posix_memalign(&a, 4096, 12345) == 0 && reinterpret_cast<uintptr_t>(a) % 4096 == 0);
    CHECK(parallax_heap_contains(a) == 1);
    free(a);
    for (int r = 0; r < 200; ++r) {  // churn: grow and shrink many vectors
        std::vector<std::vector<double>> vv;
        for (int i = 0; i < 50; ++i) vv.emplace_back((size_t)((r * 37 + i * 101) % 5000) + 1, 1.5);
        vv.erase(vv.begin() + 10, vv.begin() + 30);
        for (auto& x : vv) x.resize(x.size() * 2 + 3);
    }
    m.clear();
    v.clear();
    v.shrink_to_fit();
    CHECK(px_pool_check() == 1);
    CHECK(px_pool_high_water() > 0 && px_pool_high_water() <= px_pool_reservation());
    int on_stack = 0;
    CHECK(parallax_heap_contains(&on_stack) == 0);
    printf("ok %zu\n", px_pool_high_water());
    return 0;
}
