// CPU oracle for the parallax primitive hot path. TEST INFRASTRUCTURE ONLY: it is called
// by the tests, by smoke() as the checker, and by bench.py's CPU baseline leg; the
// runtime library never links or calls it.
//
// It restates, on the host, what each primitive must compute. Integer and ordering
// results follow the ISO semantics of the reference's host fallbacks in
// include/parallax/stdpar.hpp (parallax-runtime):
//   reduce            stdpar.hpp:146-148   (left fold; integers here wrap in unsigned)
//   inclusive_scan    stdpar.hpp:209-210
//   exclusive_scan    stdpar.hpp:237-238
//   sort              stdpar.hpp:178       (std::sort; floats ordered by the IEEE total
//                                           order, one of the orders std::sort may give)
//   copy_if           stdpar.hpp:319-321
//   remove_if         stdpar.hpp:343-345
//   partition         stdpar.hpp:369-370   (std::partition is unstable; the contract here
//                                           is the stable order of the reference's GPU
//                                           scatter, shaders/scatter.comp:15-22 and
//                                           src/kernel/kernel_launcher.cpp:1780-1781, i.e.
//                                           std::stable_partition)
//   unique            stdpar.hpp:392-393
//   argminmax / find / mismatch   src/kernel/kernel_launcher.cpp:987-1278 (first index
//                                 of the extremum / match, `count` when none)
// The modulo predicate x % m == r follows C (the remainder takes the sign of x) with m and
// r converted to the element type; x % -1 is taken as 0 (C leaves MIN % -1 undefined).
// Floating-point sums and prefixes are computed in fp64 with Neumaier compensation, the
// reference against which fp32 results are held to 1e-5 and fp64 results to 1e-12
// relative error (the fallback's own fp32 left fold stalls at 2^24 and is not used).
// Inputs come from a counter-based generator, u(seed, i) = splitmix64(seed*G + i), so the
// GPU tests, this oracle and the CPU baseline see the same data at any size.
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <vector>

#define OX extern "C" __attribute__((visibility("default")))

namespace {

inline uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}
inline uint64_t u_at(uint64_t seed, uint64_t i) {
    return splitmix64(seed * 0x9E3779B97F4A7C15ull + i);
}

// Neumaier-compensated fp64 accumulator.
struct Neumaier {
    double s = 0.0, c = 0.0;
    void add(double x) {
        double t = s + x;
        if (std::fabs(s) >= std::fabs(x)) c += (s - t) + x;
        else c += (x - t) + s;
        s = t;
    }
    double value() const { return s + c; }
};

// predicate kinds, same numbering as the runtime's Pred
enum PK { P_NONE = 0, P_GT, P_GE, P_LT, P_LE, P_EQ, P_NE, P_MOD, P_NONZERO };

// The operand is converted to the element type, as the runtime does: integer element
// types take it from the exact 64-bit integer `ci`, floating types from `c`.
template <typename T>
bool pred_eval(int kind, double c, int64_t ci, int64_t m, int64_t r, T x) {
    T cc = std::is_integral<T>::value ? (T)ci : (T)c;
    switch (kind) {
        case P_GT: return x > cc;
        case P_GE: return x >= cc;
        case P_LT: return x < cc;
        case P_LE: return x <= cc;
        case P_EQ: return x == cc;
        case P_NE: return x != cc;
        case P_NONZERO: return x != T(0);
        case P_MOD:
            if constexpr (std::is_integral<T>::value) {
                // x % -1 is 0; the C expression overflows (traps) for the minimum value
                if (std::is_signed<T>::value && (T)m == T(-1)) return T(0) == (T)r;
                return x % (T)m == (T)r;
            } else {
                return false;
            }
        default: return false;
    }
}

template <typename T>
struct Bits;
template <> struct Bits<float> { using U = uint32_t; };
template <> struct Bits<double> { using U = uint64_t; };

// IEEE total-order key (negative: flip all bits, else flip the sign bit).
template <typename F>
typename Bits<F>::U total_key(F f) {
    using U = typename Bits<F>::U;
    U b;
    memcpy(&b, &f, sizeof b);
    const U sign = U(1) << (sizeof(U) * 8 - 1);
    return (b & sign) ? ~b : (b | sign);
}

}  // namespace

// ---- generators (seeded, counter-based) ------------------------------------------------
OX void ox_gen_u64(uint64_t seed, uint64_t start, uint64_t n, uint64_t* out) {
    for (uint64_t i = 0; i < n; ++i) out[i] = u_at(seed, start + i);
}
OX void ox_gen_f32_unit(uint64_t seed, uint64_t n, float* out) {
    for (uint64_t i = 0; i < n; ++i) out[i] = (float)((double)(u_at(seed, i) >> 40) * 0x1p-24);
}
OX void ox_gen_f64_unit(uint64_t seed, uint64_t n, double* out) {
    for (uint64_t i = 0; i < n; ++i) out[i] = (double)(u_at(seed, i) >> 11) * 0x1p-53;
}
OX void ox_gen_i32_pm1000(uint64_t seed, uint64_t n, int32_t* out) {
    for (uint64_t i = 0; i < n; ++i) out[i] = (int32_t)(u_at(seed, i) % 2001) - 1000;
}
OX void ox_gen_u32_full(uint64_t seed, uint64_t n, uint32_t* out) {
    for (uint64_t i = 0; i < n; ++i) out[i] = (uint32_t)u_at(seed, i);
}
OX void ox_gen_i64_full(uint64_t seed, uint64_t n, int64_t* out) {
    for (uint64_t i = 0; i < n; ++i) out[i] = (int64_t)u_at(seed, i);
}

// ---- reduce --------------------------------------------------------------------------------
OX double ox_sum_f32(const float* x, uint64_t n) {
    Neumaier a;
    for (uint64_t i = 0; i < n; ++i) a.add((double)x[i]);
    return a.value();
}
OX double ox_sum_f64(const double* x, uint64_t n) {
    Neumaier a;
    for (uint64_t i = 0; i < n; ++i) a.add(x[i]);
    return a.value();
}
OX uint32_t ox_sum_u32(const uint32_t* x, uint64_t n) {  // also int32 (two's complement)
    uint32_t s = 0;
    for (uint64_t i = 0; i < n; ++i) s += x[i];
    return s;
}
OX uint64_t ox_sum_u64(const uint64_t* x, uint64_t n) {  // also int64
    uint64_t s = 0;
    for (uint64_t i = 0; i < n; ++i) s += x[i];
    return s;
}

template <typename T>
static T minmax_t(const T* x, uint64_t n, int want_max) {
    T best = x[0];
    for (uint64_t i = 1; i < n; ++i) best = want_max ? (x[i] > best ? x[i] : best)
                                                     : (x[i] < best ? x[i] : best);
    return best;
}
OX float ox_minmax_f32(const float* x, uint64_t n, int mx) { return minmax_t(x, n, mx); }
OX double ox_minmax_f64(const double* x, uint64_t n, int mx) { return minmax_t(x, n, mx); }
OX int32_t ox_minmax_i32(const int32_t* x, uint64_t n, int mx) { return minmax_t(x, n, mx); }
OX int64_t ox_minmax_i64(const int64_t* x, uint64_t n, int mx) { return minmax_t(x, n, mx); }
OX uint32_t ox_minmax_u32(const uint32_t* x, uint64_t n, int mx) { return minmax_t(x, n, mx); }
OX uint64_t ox_minmax_u64(const uint64_t* x, uint64_t n, int mx) { return minmax_t(x, n, mx); }

// ---- scans -----------------------------------------------------------------------------------
// fp: compensated fp64 prefix written as double (exclusive when excl != 0, with init).
OX void ox_scan_f32(const float* x, double* out, uint64_t n, int excl, double init) {
    Neumaier a;
    a.add(excl ? init : 0.0);
    for (uint64_t i = 0; i < n; ++i) {
        if (excl) { out[i] = a.value(); a.add((double)x[i]); }
        else { a.add((double)x[i]); out[i] = a.value(); }
    }
}
OX void ox_scan_f64(const double* x, double* out, uint64_t n, int excl, double init) {
    Neumaier a;
    a.add(excl ? init : 0.0);
    for (uint64_t i = 0; i < n; ++i) {
        if (excl) { out[i] = a.value(); a.add(x[i]); }
        else { a.add(x[i]); out[i] = a.value(); }
    }
}
OX void ox_scan_u32(const uint32_t* x, uint32_t* out, uint64_t n, int excl, uint32_t init) {
    uint32_t s = excl ? init : 0u;
    for (uint64_t i = 0; i < n; ++i) {
        if (excl) { out[i] = s; s += x[i]; }
        else { s += x[i]; out[i] = s; }
    }
}
OX void ox_scan_u64(const uint64_t* x, uint64_t* out, uint64_t n, int excl, uint64_t init) {
    uint64_t s = excl ? init : 0u;
    for (uint64_t i = 0; i < n; ++i) {
        if (excl) { out[i] = s; s += x[i]; }
        else { s += x[i]; out[i] = s; }
    }
}

// ---- sort ---------------------------------------------------------------------------------------
OX void ox_sort_u32(uint32_t* x, uint64_t n) { std::sort(x, x + n); }
OX void ox_sort_u64(uint64_t* x, uint64_t n) { std::sort(x, x + n); }
OX void ox_sort_i32(int32_t* x, uint64_t n) { std::sort(x, x + n); }
OX void ox_sort_i64(int64_t* x, uint64_t n) { std::sort(x, x + n); }
OX void ox_sort_f32(float* x, uint64_t n) {
    std::sort(x, x + n, [](float a, float b) { return total_key(a) < total_key(b); });
}
OX void ox_sort_f64(double* x, uint64_t n) {
    std::sort(x, x + n, [](double a, double b) { return total_key(a) < total_key(b); });
}

// ---- compaction -----------------------------------------------------------------------------------
// mode 0 copy_if, 1 remove_if, 2 stable partition, 3 unique. Returns the kept count
// (partition: the number of elements satisfying the predicate; all n are written).
template <typename T>
static uint64_t compact_t(const T* in, T* out, uint64_t n, int mode, int kind, double c, int64_t ci,
                          int64_t m, int64_t r) {
    uint64_t k = 0;
    if (mode == 3) {
        for (uint64_t i = 0; i < n; ++i)
            if (i == 0 || !(in[i] == in[i - 1])) out[k++] = in[i];
        return k;
    }
    if (mode == 2) {
        std::vector<T> rest;
        for (uint64_t i = 0; i < n; ++i) {
            if (pred_eval<T>(kind, c, ci, m, r, in[i])) out[k++] = in[i];
            else rest.push_back(in[i]);
        }
        std::copy(rest.begin(), rest.end(), out + k);
        return k;
    }
    for (uint64_t i = 0; i < n; ++i) {
        bool p = pred_eval<T>(kind, c, ci, m, r, in[i]);
        if (mode == 1) p = !p;
        if (p) out[k++] = in[i];
    }
    return k;
}
#define OX_COMPACT(sfx, T)                                                                   \
    OX uint64_t ox_compact_##sfx(const T* in, T* out, uint64_t n, int mode, int kind,          \
                                 double c, int64_t ci, int64_t m, int64_t r) {                 \
        return compact_t<T>(in, out, n, mode, kind, c, ci, m, r);                              \
    }                                                                                          \
    OX uint64_t ox_count_##sfx(const T* in, uint64_t n, int kind, double c, int64_t ci,       \
                               int64_t m, int64_t r) {                                         \
        uint64_t k = 0;                                                                        \
        for (uint64_t i = 0; i < n; ++i) k += pred_eval<T>(kind, c, ci, m, r, in[i]);              \
        return k;                                                                              \
    }                                                                                          \
    OX uint64_t ox_find_##sfx(const T* in, uint64_t n, int kind, double c, int64_t ci,        \
                              int64_t m, int64_t r, int negate) {                              \
        for (uint64_t i = 0; i < n; ++i)                                                       \
            if (pred_eval<T>(kind, c, ci, m, r, in[i]) != (negate != 0)) return i;                 \
        return n;                                                                              \
    }                                                                                          \
    OX uint64_t ox_argminmax_##sfx(const T* in, uint64_t n, int want_max, int want_last) {    \
        if (n <= 1) return 0;                                                                  \
        uint64_t b = 0;                                                                        \
        for (uint64_t i = 1; i < n; ++i) {                                                     \
            bool better = want_max ? in[i] > in[b] : in[i] < in[b];                            \
            bool equal = !(in[i] < in[b]) && !(in[b] < in[i]);                                 \
            if (better || (equal && want_last)) b = i;                                         \
        }                                                                                      \
        return b;                                                                              \
    }                                                                                          \
    OX uint64_t ox_mismatch_##sfx(const T* a, const T* b, uint64_t n) {                       \
        for (uint64_t i = 0; i < n; ++i)                                                       \
            if (!(a[i] == b[i])) return i;                                                     \
        return n;                                                                              \
    }
OX_COMPACT(f32, float)
OX_COMPACT(f64, double)
OX_COMPACT(i32, int32_t)
OX_COMPACT(i64, int64_t)
OX_COMPACT(u32, uint32_t)
OX_COMPACT(u64, uint64_t)

// ---- map with captures and relocation ---------------------------------------------------------------
// Records {float x; uint32 pad; uint64 p}, p a HOST address in [host_base, ...) of `tgt`
// (host copy): y[i] = a*x + *p, rounded in fp32 per operation.
OX void ox_saxpy_gather(const void* records, uint64_t n, float a, const float* tgt,
                        uint64_t host_base, float* y) {
    const unsigned char* r = static_cast<const unsigned char*>(records);
    for (uint64_t i = 0; i < n; ++i) {
        float x;
        uint64_t p;
        memcpy(&x, r + 16 * i, 4);
        memcpy(&p, r + 16 * i + 8, 8);
        volatile float ax = a * x;  // keep the product rounded to fp32 (no contraction)
        y[i] = ax + tgt[(p - host_base) / 4];
    }
}
