// Drives the reference's own stdpar funnels (include/parallax/stdpar.hpp, unmodified) on
// seeded inputs and writes every result to a file. TEST INFRASTRUCTURE ONLY.
//
// oracle/Makefile builds it three times from the same source:
//   _ref/stdpar_driver_gpu   linked against libparallax-runtime.so: fixed funnels (reduce,
//                            scans, sort, unique) resolve to the built-in sm_100a kernels;
//                            the functor funnels resolve to the sm_100a images this program
//                            registers at start-up, the way compiler-emitted registrars do
//                            (include/parallax/runtime.h:96-103);
//   _ref/stdpar_driver_heap  the same, also linked with the whole-heap capture shim
//                            (lib/libparallax-heap.a): every std::vector lives in the heap
//                            pool, so the funnels find their data in the arena and call the
//                            runtime on it in place, and a transform may chase pointers
//                            stored in heap records;
//   _ref/stdpar_driver_host  linked against abi_stub.cpp, whose lookups all miss: every call
//                            runs the reference's host fallback.
// tests/test_gpu_stdpar.py runs both and compares them call by call.
//
//   stdpar_driver <image dir> <output file>
//
// Output: one record per call: name (NUL-terminated), uint64 runtime launches the call
// issued (0 where the runtime is absent), uint64 scalar result (reduce bits, kept count,
// partition point, count), uint64 byte count, then that many bytes of the output array.
// Inputs are u(seed, i) = splitmix64(seed * 0x9E3779B97F4A7C15 + i), the oracle's generator.
#include <parallax/stdpar.hpp>

#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <functional>
#include <string>
#include <vector>

// The runtime's launch counter (runtime_ext.h); absent in the host build.
extern "C" uint64_t parallax_launch_count(void) __attribute__((weak));

// Functors at namespace scope: their names appear in the funnel keys as written here.
struct KeepMod3 { bool operator()(int x) const { return x % 3 == 0; } };
struct Neg { bool operator()(int x) const { return x < 0; } };
struct GtHalf { bool operator()(float x) const { return x > 0.5f; } };
struct HalfD { double operator()(int x) const { return (double)x * 0.5; } };
struct Affine {  // captures: two floats
    float a, b;
    void operator()(float& x) const {
        volatile float ax = a * x;  // rounded product, then a rounded sum (no contraction)
        x = ax + b;
    }
};
struct Rec {  // a heap record holding a pointer into another heap array
    float x;
    unsigned pad;
    const float* p;
};
struct GatherPlus {  // y = 0 * x + *p (the gather image with no captures: a = 0)
    float operator()(const Rec& r) const {
        volatile float ax = 0.0f * r.x;
        return ax + *r.p;
    }
};
struct AffineDefault {  // no captures: x = 2x + 1
    void operator()(float& x) const {
        volatile float ax = 2.0f * x;
        x = ax + 1.0f;
    }
};

namespace {

uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}
uint64_t u_at(uint64_t seed, uint64_t i) { return splitmix64(seed * 0x9E3779B97F4A7C15ull + i); }

std::vector<float> f32_unit(uint64_t seed, size_t n) {
    std::vector<float> v(n);
    for (size_t i = 0; i < n; ++i) v[i] = (float)((double)(u_at(seed, i) >> 40) * 0x1p-24);
    return v;
}
std::vector<double> f64_unit(uint64_t seed, size_t n) {
    std::vector<double> v(n);
    for (size_t i = 0; i < n; ++i) v[i] = (double)(u_at(seed, i) >> 11) * 0x1p-53;
    return v;
}
std::vector<int> i32_pm1000(uint64_t seed, size_t n) {
    std::vector<int> v(n);
    for (size_t i = 0; i < n; ++i) v[i] = (int)(u_at(seed, i) % 2001) - 1000;
    return v;
}
std::vector<long> i64_full(uint64_t seed, size_t n) {
    std::vector<long> v(n);
    for (size_t i = 0; i < n; ++i) v[i] = (long)u_at(seed, i);
    return v;
}
std::vector<unsigned> u32_full(uint64_t seed, size_t n) {
    std::vector<unsigned> v(n);
    for (size_t i = 0; i < n; ++i) v[i] = (unsigned)u_at(seed, i);
    return v;
}

FILE* g_out = nullptr;

uint64_t launches() { return parallax_launch_count ? parallax_launch_count() : 0; }

template <typename T>
void record(const std::string& name, uint64_t before, uint64_t scalar, const T* data, size_t n);
void record_scalar(const std::string& name, uint64_t before, uint64_t scalar) {
    static const char none = 0;
    record(name, before, scalar, &none, 0);
}
template <typename T>
void record(const std::string& name, uint64_t before, uint64_t scalar, const T* data, size_t n) {
    const uint64_t l = launches() - before;
    const uint64_t bytes = n * sizeof(T);
    fwrite(name.c_str(), 1, name.size() + 1, g_out);
    fwrite(&l, 8, 1, g_out);
    fwrite(&scalar, 8, 1, g_out);
    fwrite(&bytes, 8, 1, g_out);
    if (bytes && data) fwrite(data, 1, bytes, g_out);
}
template <typename T>
uint64_t bits(T v) {
    uint64_t b = 0;
    memcpy(&b, &v, sizeof v);
    return b;
}

// Images this program registers (their fatbins live in <image dir>), keyed exactly as GCC
// spells the funnels' __PRETTY_FUNCTION__.
const char* const SZ = "; std::size_t = long unsigned int]";
std::vector<std::vector<unsigned>> g_images;  // registered images must outlive the process

bool register_image(const std::string& dir, const std::string& key, const char* image) {
    const std::string path = dir + "/" + image + ".fatbin";
    FILE* f = fopen(path.c_str(), "rb");
    if (!f) {
        fprintf(stderr, "stdpar_driver: cannot open %s\n", path.c_str());
        return false;
    }
    std::vector<unsigned char> bytes;
    unsigned char buf[65536];
    size_t got;
    while ((got = fread(buf, 1, sizeof buf, f)) > 0) bytes.insert(bytes.end(), buf, buf + got);
    fclose(f);
    std::vector<unsigned> words((bytes.size() + 3) / 4, 0u);
    memcpy(words.data(), bytes.data(), bytes.size());
    g_images.push_back(std::move(words));
    parallax_kernel_register(strdup(key.c_str()), g_images.back().data(), g_images.back().size());
    return true;
}

bool register_all(const std::string& dir) {
    const std::string cpy = "std::size_t parallax::detail::device_copy_if(const T*, T*, std::size_t, Pred) [with T = int; Pred = KeepMod3";
    const std::string rem = "std::size_t parallax::detail::device_remove_if(T*, std::size_t, Pred) [with T = int; Pred = KeepMod3";
    const std::string par = "std::size_t parallax::detail::device_partition(T*, std::size_t, Pred) [with T = int; Pred = Neg";
    const std::string inv = "void parallax::detail::device_invoke(T*, std::size_t, F) [with T = float; F = ";
    const std::string xf = "void parallax::detail::device_transform(const Tin*, Tout*, std::size_t, F) [with Tin = int; Tout = double; F = HalfD";
    const std::string cnt = "long int parallax::detail::device_count_if(const T*, std::size_t, Pred) [with T = float; Pred = GtHalf";
    const std::string gat = "void parallax::detail::device_transform(const Tin*, Tout*, std::size_t, F) [with Tin = Rec; Tout = float; F = GatherPlus";
    const std::string trd = "U parallax::detail::device_transform_reduce(const T*, std::size_t, F) [with T = int; U = double; F = HalfD";
    bool ok = true;
    ok &= register_image(dir, cpy + SZ + ":flags", "flags_mod3_i32");
    ok &= register_image(dir, rem + SZ + ":flags", "flags_not_mod3_i32");
    ok &= register_image(dir, par + SZ + ":flags", "flags_neg_i32");
    ok &= register_image(dir, inv + "Affine" + SZ, "affine_f32");
    ok &= register_image(dir, inv + "AffineDefault" + SZ, "affine_f32");
    ok &= register_image(dir, xf + SZ, "half_i32_to_f64");
    // transforms that also export their element function (LTO-IR): the runtime fuses each
    // funnel's transform + reduce into one pass
    ok &= register_image(dir, cnt + SZ + ":pred", "pred_gt_half_f32_lto");
    ok &= register_image(dir, trd + SZ + ":xform", "xform_half_i32_to_f64_lto");
    ok &= register_image(dir, gat + SZ, "saxpy_gather_f32");
    return ok;
}

void run(size_t n) {
    const std::string sfx = "@" + std::to_string(n);
    const auto P = parallax::par;
    uint64_t b;
    {  // reduce (init 0; the funnel adds init on the host)
        auto f = f32_unit(21, n);
        b = launches();
        float r = parallax::reduce(P, f.begin(), f.end(), 0.0f);
        record_scalar("reduce_f32" + sfx, b, bits(r));
        auto d = f64_unit(22, n);
        b = launches();
        double rd = parallax::reduce(P, d.begin(), d.end(), 0.0);
        record_scalar("reduce_f64" + sfx, b, bits(rd));
        auto i = i32_pm1000(23, n);
        b = launches();
        int ri = parallax::reduce(P, i.begin(), i.end(), 0);
        record_scalar("reduce_i32" + sfx, b, bits(ri));
        auto l = i64_full(24, n);
        b = launches();
        long rl = parallax::reduce(P, l.begin(), l.end(), 0L);
        record_scalar("reduce_i64" + sfx, b, bits(rl));
    }
    {  // scans
        auto f = f32_unit(21, n);
        std::vector<float> fo(n);
        b = launches();
        parallax::inclusive_scan(P, f.begin(), f.end(), fo.begin());
        record("inclusive_scan_f32" + sfx, b, 0, fo.data(), n);
        auto l = i64_full(24, n);
        std::vector<long> lo(n);
        b = launches();
        parallax::inclusive_scan(P, l.begin(), l.end(), lo.begin());
        record("inclusive_scan_i64" + sfx, b, 0, lo.data(), n);
        auto i = i32_pm1000(23, n);
        std::vector<int> io(n);
        b = launches();
        parallax::exclusive_scan(P, i.begin(), i.end(), io.begin(), 5);
        record("exclusive_scan_i32" + sfx, b, 0, io.data(), n);
        auto d = f64_unit(22, n);
        std::vector<double> dout(n);
        b = launches();
        parallax::exclusive_scan(P, d.begin(), d.end(), dout.begin(), 0.25);
        record("exclusive_scan_f64" + sfx, b, 0, dout.data(), n);
    }
    {  // sorts
        auto u = u32_full(25, n);
        b = launches();
        parallax::sort(P, u.begin(), u.end());
        record("sort_u32" + sfx, b, 0, u.data(), n);
        auto f = f32_unit(26, n);
        for (auto& v : f) v = v * 2.0f - 1.0f;
        for (size_t i = 0; i < n / 50; ++i) f[i] = f[i + n / 2];  // exact duplicates
        if (n > 3) f[1] = 0.0f, f[3] = -0.0f;
        b = launches();
        parallax::sort(P, f.begin(), f.end());
        record("sort_f32" + sfx, b, 0, f.data(), n);
    }
    {  // unique over sorted values
        auto u = u32_full(27, n);
        std::vector<int> v(n);
        for (size_t i = 0; i < n; ++i) v[i] = (int)(u[i] % 5000u);
        std::sort(v.begin(), v.end());
        b = launches();
        auto e = parallax::unique(P, v.begin(), v.end());
        const size_t k = (size_t)(e - v.begin());
        record("unique_i32" + sfx, b, k, v.data(), k);
    }
    {  // compaction with registered predicate images
        auto x = i32_pm1000(23, n);
        std::vector<int> o(n, -7);
        b = launches();
        auto e = parallax::copy_if(P, x.begin(), x.end(), o.begin(), KeepMod3{});
        size_t k = (size_t)(e - o.begin());
        record("copy_if_mod3_i32" + sfx, b, k, o.data(), k);
        auto r = x;
        b = launches();
        auto re = parallax::remove_if(P, r.begin(), r.end(), KeepMod3{});
        k = (size_t)(re - r.begin());
        record("remove_if_mod3_i32" + sfx, b, k, r.data(), k);
        auto q = x;
        b = launches();
        auto pe = parallax::partition(P, q.begin(), q.end(), Neg{});
        k = (size_t)(pe - q.begin());
        record("partition_neg_i32" + sfx, b, k, q.data(), n);
    }
    {  // element-wise funnels with registered images
        auto f = f32_unit(21, n);
        b = launches();
        parallax::for_each(P, f.begin(), f.end(), Affine{1.5f, -0.25f});
        record("for_each_affine_f32" + sfx, b, 0, f.data(), n);
        auto g = f32_unit(21, n);
        b = launches();
        parallax::for_each(P, g.begin(), g.end(), AffineDefault{});
        record("for_each_default_f32" + sfx, b, 0, g.data(), n);
        auto i = i32_pm1000(23, n);
        std::vector<double> d(n);
        b = launches();
        parallax::transform(P, i.begin(), i.end(), d.begin(), HalfD{});
        record("transform_half_i32" + sfx, b, 0, d.data(), n);
        auto c = f32_unit(21, n);
        b = launches();
        long cnt = parallax::count_if(P, c.begin(), c.end(), GtHalf{});
        record_scalar("count_if_gt_half_f32" + sfx, b, (uint64_t)cnt);
        auto t = i32_pm1000(24, n);
        b = launches();
        const double tr = parallax::transform_reduce(P, t.begin(), t.end(), 0.0, std::plus<>{},
                                                     HalfD{});
        uint64_t tr_bits;
        memcpy(&tr_bits, &tr, sizeof tr_bits);
        record_scalar("transform_reduce_half_i32" + sfx, b, tr_bits);
    }
    {  // where the heap lives, and a transform that chases pointers stored in heap records
        std::vector<float> tgt = f32_unit(28, n);
        const uint64_t where = (uint64_t)parallax_heap_contains(tgt.data()) |
                               (uint64_t)parallax_arena_contains(tgt.data()) << 1;
        record_scalar("heap_capture" + sfx, launches(), where);
        // Stored pointers mean something on the device only when the heap is captured (the
        // host fallback follows them anyway); without capture the call is left out.
        const bool host_build = parallax_launch_count == nullptr;
        if (host_build || where == 3) {
            std::vector<Rec> recs(n);
            for (size_t i = 0; i < n; ++i)
                recs[i] = Rec{(float)(u_at(29, i) >> 40) * 0x1p-24f, 0u, &tgt[u_at(30, i) % n]};
            std::vector<float> y(n);
            b = launches();
            parallax::transform(P, recs.begin(), recs.end(), y.begin(), GatherPlus{});
            record("transform_gather_f32" + sfx, b, 0, y.data(), n);
        }
    }
}

}  // namespace

int main(int argc, char** argv) {
    if (argc != 3) {
        fprintf(stderr, "usage: %s <image dir> <output file>\n", argv[0]);
        return 2;
    }
    if (!register_all(argv[1])) return 3;
    g_out = fopen(argv[2], "wb");
    if (!g_out) return 4;
    for (size_t n : {size_t(1), size_t(1000), size_t(300007)}) run(n);
    fclose(g_out);
    return 0;
}
