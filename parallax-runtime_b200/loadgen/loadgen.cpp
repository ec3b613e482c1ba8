// Load generator for the serving mix: many host threads issue Poisson-arrival primitive
// requests against the parallax C ABI, either one synchronous call per request (the
// per-call path) or through the serving loop (parallax_serve_submit / _wait). It uses only
// the public ABI (include/parallax/runtime.h, runtime_ext.h) and is built as its own
// library, libparallax-loadgen.so, next to the runtime.
//
// Mix (per request, from a per-thread seeded generator): operation 40 % reduce (sum),
// 30 % exclusive scan, 20 % sort, 10 % copy_if; element type uniform over fp32 / fp64 /
// int32 / int64; n = floor(2^u), u uniform in [log2_min, log2_max]. Inputs of reduce,
// scan and copy_if are windows at random 256-byte-aligned offsets of one shared 2^26-element
// array per type (1.5 GiB in all, far above the 126 MB L2) in device-resident arena blocks.
// Outputs and the sort's data are arena blocks allocated for the request when it is issued
// and freed when it completes (a request waits for its thread's oldest one when the arena is
// full). Sort requests sort whatever the freshly allocated block holds (earlier requests'
// bytes); this measures time only, results are checked by the tests.
// With `warmup`, each client first runs one largest request of each operation untimed (so
// per-thread and per-lane buffers that grow on first use are in place), then all clients
// start one shared measured window.
// Latency = completion - arrival time. The per-call path issues a thread's requests in
// order, so a request that arrives while its thread is busy waits, as it would in a client
// with one connection; the served path submits at arrival and collects completions on a
// second thread (mode 1) or on the same thread by polling (mode 4), with at most
// `max_inflight` outstanding requests per client.
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>
#include <time.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <thread>
#include <vector>

#include "parallax/runtime.h"
#include "parallax/runtime_ext.h"

#define LG_EXPORT extern "C" __attribute__((visibility("default")))

extern "C" {
typedef struct px_loadgen_config {
    uint32_t threads;        /* client threads (16) */
    uint32_t mode;           /* 0 per-call, 1 served, 2 per-call serialized by one lock
                                (one call at a time, as a runtime that is not thread-safe
                                must be driven), 3 device bound: every thread enqueues its
                                calls asynchronously on its own stream and synchronizes once
                                per 64 calls, so the rate is what the device sustains for the
                                mix with no host round trip per request (latencies are not
                                meaningful in this mode), 4 served with one thread per client
                                (submissions and parallax_serve_poll of the oldest outstanding
                                request on the same thread) */
    double rate;             /* offered requests/s over all threads; <= 0: back-to-back */
    double seconds;          /* issuing window */
    uint64_t seed;
    uint32_t log2_min, log2_max;
    uint32_t max_inflight;   /* served mode: outstanding requests per thread (64) */
    uint32_t warmup;         /* nonzero: every thread first runs one largest request of each
                                operation (fp64), untimed, so buffers grown on first use are
                                in place before the measured window */
} px_loadgen_config;

typedef struct px_loadgen_result {
    uint64_t completed, errors;
    double seconds;          /* first arrival to last completion */
    double req_s, p50_ms, p99_ms, mean_ms, max_ms;
    double gbytes;           /* algorithmic bytes of the completed requests */
    double gb_s;
    uint64_t per_op[4];      /* completed reduce / scan / sort / copy_if */
} px_loadgen_result;
}

namespace {

constexpr uint64_t kPoolElems = 1ull << 26;
const char* kTypes[4] = {"f32", "f64", "i32", "i64"};
const size_t kSize[4] = {4, 8, 4, 8};

uint64_t now_ns() {
    timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (uint64_t)ts.tv_sec * 1000000000ull + (uint64_t)ts.tv_nsec;
}

uint64_t splitmix(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

struct Rng {
    uint64_t s;
    uint64_t next() { return splitmix(s++); }
    double unit() { return (double)(next() >> 11) * 0x1p-53; }
};

struct Pool {
    void* in[4] = {nullptr, nullptr, nullptr, nullptr};
    parallax_kernel_t reduce[4], scan[4], sort[4], copy_if[4];
    bool ready = false;
} g_pool;

enum Op { OP_REDUCE = 0, OP_SCAN = 1, OP_SORT = 2, OP_COPY_IF = 3 };

struct Item {
    int op = 0, t = 0;
    uint64_t n = 0;
    uint64_t arrival = 0, done = 0;
    uint64_t in_off = 0;
    void* buf = nullptr;       // arena block: scan / copy_if output or the sort's data
    uint64_t result = 0;       // reduce value / kept count
    uint64_t ticket = 0;
    int status = 0;
};

Item make_item(Rng& r, const px_loadgen_config& c) {
    Item it;
    const double u = r.unit() * 100.0;
    it.op = u < 40 ? OP_REDUCE : u < 70 ? OP_SCAN : u < 90 ? OP_SORT : OP_COPY_IF;
    it.t = (int)(r.next() % 4);
    const double e = c.log2_min + r.unit() * (c.log2_max - c.log2_min);
    it.n = std::max<uint64_t>(1, (uint64_t)floor(pow(2.0, e)));
    if (it.n > kPoolElems) it.n = kPoolElems;
    const uint64_t span = kPoolElems - it.n;
    const uint64_t per256 = 256 / kSize[it.t];
    it.in_off = span ? (r.next() % (span + 1)) / per256 * per256 : 0;
    return it;
}

uint64_t alg_bytes(const Item& it) {
    const uint64_t s = kSize[it.t];
    switch (it.op) {
        case OP_REDUCE: return it.n * s;
        case OP_COPY_IF: return (it.n + it.result) * s;
        default: return 2 * it.n * s;
    }
}

const void* input_of(const Item& it) {
    return static_cast<const char*>(g_pool.in[it.t]) + it.in_off * kSize[it.t];
}

bool alloc_buf(Item& it) {
    if (it.op == OP_REDUCE) return true;
    const size_t bytes = std::max<size_t>(it.n * kSize[it.t], 256);
    it.buf = parallax_arena_alloc(bytes, 256);
    if (!it.buf) return false;
    parallax_arena_set_residency(it.buf, PARALLAX_DEVICE_RESIDENT);
    return true;
}

void free_buf(Item& it) {
    if (it.buf) parallax_arena_free(it.buf);
    it.buf = nullptr;
}

// ---- per-call path: one synchronous ABI call ---------------------------------------------
std::mutex g_call_mu;  // mode 2: one call at a time

// `dev_result`: where a reduce writes its value in async mode (a device-resident block).
int run_call(Item& it, void* dev_result = nullptr) {
    const int t = it.t;
    const size_t s = kSize[t];
    parallax_clear_error();
    switch (it.op) {
        case OP_REDUCE:
            parallax_reduce(g_pool.reduce[t], const_cast<void*>(input_of(it)), it.n, s,
                            dev_result ? dev_result : &it.result);
            break;
        case OP_SCAN: {
            const uint64_t zero = 0;
            parallax_kernel_t h = g_pool.scan[t];
            parallax_exclusive_scan(h, h, h, const_cast<void*>(input_of(it)), it.buf, it.n, s, &zero);
            break;
        }
        case OP_SORT:
            parallax_sort(g_pool.sort[t], it.buf, it.n, s);
            break;
        default: {
            parallax_kernel_t h = g_pool.copy_if[t];
            it.result = parallax_copy_if(h, h, h, h, const_cast<void*>(input_of(it)), it.buf, it.n, s,
                                         t < 2);
            if (dev_result) it.result = 0;  // async: the count is not read back
            break;
        }
    }
    return parallax_last_error();
}

// ---- served path ------------------------------------------------------------------------------
int submit(Item& it) {
    static const uint64_t zero = 0;
    parallax_request q;
    memset(&q, 0, sizeof q);
    q.count = it.n;
    q.result = &it.result;
    switch (it.op) {
        case OP_REDUCE:
            q.kernel = g_pool.reduce[it.t];
            q.input = input_of(it);
            break;
        case OP_SCAN:
            q.kernel = g_pool.scan[it.t];
            q.input = input_of(it);
            q.output = it.buf;
            q.init = &zero;
            q.flags = PARALLAX_REQ_EXCLUSIVE;
            break;
        case OP_SORT:
            q.kernel = g_pool.sort[it.t];
            q.input = it.buf;
            break;
        default:
            q.kernel = g_pool.copy_if[it.t];
            q.input = input_of(it);
            q.output = it.buf;
            break;
    }
    return parallax_serve_submit(&q, &it.ticket);
}

void sleep_until(uint64_t t) {
    for (;;) {
        const uint64_t n = now_ns();
        if (n >= t) return;
        const uint64_t d = t - n;
        if (d > 200000) std::this_thread::sleep_for(std::chrono::nanoseconds(d - 100000));
        else std::this_thread::yield();
    }
}

struct ThreadOut {
    std::vector<Item> items;
};

// Start line: every client finishes its warm-up, then all share one measured window.
struct StartLine {
    std::mutex mu;
    std::condition_variable cv;
    uint32_t arrived = 0, expected = 0;
    uint64_t t0 = 0, t_end = 0;
    double seconds = 0;
    void arrive_and_wait(uint64_t* t0_out, uint64_t* t_end_out) {
        std::unique_lock<std::mutex> lk(mu);
        if (++arrived == expected) {
            t0 = now_ns() + 2000000;  // 2 ms for the clients to wake
            t_end = t0 + (uint64_t)(seconds * 1e9);
            cv.notify_all();
        } else {
            cv.wait(lk, [&] { return arrived == expected; });
        }
        *t0_out = t0;
        *t_end_out = t_end;
    }
};

void warm_up(const px_loadgen_config& c) {
    for (int op = 0; op < 4; ++op) {
        Item it;
        it.op = op;
        it.t = 1;  // fp64: the largest buffers
        it.n = std::min<uint64_t>(1ull << c.log2_max, kPoolElems);
        while (!alloc_buf(it)) std::this_thread::yield();
        if (c.mode != 1 && c.mode != 4) {
            run_call(it);
        } else if (submit(it) == PARALLAX_OK) {
            parallax_serve_wait(it.ticket, nullptr);
        }
        free_buf(it);
    }
}

void client(const px_loadgen_config& c, int tid, StartLine* line, ThreadOut* out) {
    if (c.warmup) warm_up(c);
    uint64_t t0, t_end;
    line->arrive_and_wait(&t0, &t_end);
    Rng r{c.seed * 1000003ull + (uint64_t)tid * 7919ull};
    const double per_thread_rate = c.rate > 0 ? c.rate / c.threads : 0.0;
    uint64_t next_arrival = t0;
    auto advance = [&] {
        if (per_thread_rate > 0) {
            const double gap = -log(1.0 - r.unit()) / per_thread_rate;
            next_arrival += (uint64_t)(gap * 1e9);
        }
    };
    advance();
    if (c.mode == 3) {
        void* dres = parallax_arena_alloc(256, 256);
        if (!dres || parallax_arena_set_residency(dres, PARALLAX_DEVICE_RESIDENT) != PARALLAX_OK) {
            Item bad;
            bad.status = PARALLAX_ERR_OUT_OF_MEMORY;
            out->items.push_back(bad);
            return;
        }
        parallax_set_async(1);
        std::vector<Item> chunk;
        auto drain = [&] {
            const int st = parallax_synchronize();
            const uint64_t t = now_ns();
            for (Item& it : chunk) {
                it.done = t;
                if (it.status == PARALLAX_OK) it.status = st;
                free_buf(it);
                out->items.push_back(it);
            }
            chunk.clear();
        };
        sleep_until(t0);
        for (;;) {
            Item it = make_item(r, c);
            it.arrival = now_ns();
            if (it.arrival >= t_end) break;
            if (!alloc_buf(it)) {  // arena full: let this thread's calls finish first
                drain();
                while (!alloc_buf(it)) std::this_thread::yield();
            }
            it.status = run_call(it, dres);
            chunk.push_back(it);
            if (chunk.size() == 64) drain();
        }
        drain();
        parallax_set_async(0);
        parallax_arena_free(dres);
        return;
    }
    if (c.mode == 0 || c.mode == 2) {
        sleep_until(t0);
        for (;;) {
            Item it = make_item(r, c);
            it.arrival = per_thread_rate > 0 ? next_arrival : now_ns();
            if (it.arrival >= t_end) break;
            sleep_until(it.arrival);
            while (!alloc_buf(it)) std::this_thread::yield();
            if (c.mode == 2) {
                std::lock_guard<std::mutex> g(g_call_mu);
                it.status = run_call(it);
            } else {
                it.status = run_call(it);
            }
            it.done = now_ns();
            free_buf(it);
            out->items.push_back(it);
            advance();
        }
        return;
    }
    if (c.mode == 4) {
        // served, one thread per client: submit at arrival while fewer than max_inflight of
        // the client's requests are outstanding, and between submissions poll the oldest
        // outstanding one (parallax_serve_poll), so no second thread waits per client. The
        // item vector never reallocates (capacity reserved up front).
        std::vector<Item>& items = out->items;
        items.reserve(1 << 16);
        std::deque<size_t> pending;
        auto collect = [&]() -> bool {  // true when the oldest outstanding request finished
            if (pending.empty()) return false;
            Item& it = items[pending.front()];
            int fin = 0;
            uint64_t done = 0;
            const int st = parallax_serve_poll(it.ticket, &fin, &done);
            if (!fin) return false;
            it.status = st;
            it.done = done;
            free_buf(it);
            pending.pop_front();
            return true;
        };
        uint32_t idle = 0;
        auto pause = [&] {
            __builtin_ia32_pause();
            if ((++idle & 255) == 0) std::this_thread::yield();
        };
        sleep_until(t0);
        Item next = make_item(r, c);
        next.arrival = per_thread_rate > 0 ? next_arrival : now_ns();
        for (;;) {
            const uint64_t now = now_ns();
            if ((per_thread_rate > 0 ? next.arrival : now) >= t_end ||
                items.size() + 1 >= items.capacity())
                break;
            if (now >= next.arrival && pending.size() < c.max_inflight) {
                if (!alloc_buf(next)) {  // arena full: wait for this client's oldest request
                    if (!collect()) pause();
                    continue;
                }
                if (per_thread_rate <= 0) next.arrival = now_ns();
                items.push_back(next);
                Item& stored = items.back();
                if (submit(stored) != PARALLAX_OK) {
                    stored.status = parallax_last_error();
                    stored.done = now_ns();
                    free_buf(stored);
                } else {
                    pending.push_back(items.size() - 1);
                }
                advance();
                next = make_item(r, c);
                next.arrival = per_thread_rate > 0 ? next_arrival : now_ns();
                continue;
            }
            if (!collect()) pause();
        }
        while (!pending.empty())
            if (!collect()) pause();
        return;
    }
    // served: submit at arrival, a waiter thread collects completions in order. The item
    // vector never reallocates (capacity reserved up front), so the waiter may hold indices.
    std::mutex mu;
    std::condition_variable cv;
    std::deque<size_t> pending;
    bool finished = false;
    std::vector<Item>& items = out->items;
    items.reserve(1 << 16);
    std::thread waiter([&] {
        for (;;) {
            size_t idx;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv.wait(lk, [&] { return finished || !pending.empty(); });
                if (pending.empty()) return;
                idx = pending.front();
            }
            Item& it = items[idx];
            uint64_t done = 0;
            it.status = parallax_serve_wait(it.ticket, &done);
            it.done = done;
            free_buf(it);
            {
                std::lock_guard<std::mutex> g(mu);
                pending.pop_front();
            }
            cv.notify_all();
        }
    });
    sleep_until(t0);
    for (;;) {
        Item it = make_item(r, c);
        it.arrival = per_thread_rate > 0 ? next_arrival : now_ns();
        if (it.arrival >= t_end || items.size() + 1 >= items.capacity()) break;
        sleep_until(it.arrival);
        {
            std::unique_lock<std::mutex> lk(mu);
            cv.wait(lk, [&] { return pending.size() < c.max_inflight; });
        }
        while (!alloc_buf(it)) {  // arena full: wait for this thread's oldest request
            std::unique_lock<std::mutex> lk(mu);
            const size_t before = pending.size();
            if (before == 0) {
                lk.unlock();
                std::this_thread::yield();
                continue;
            }
            cv.wait(lk, [&] { return pending.size() < before; });
        }
        if (per_thread_rate <= 0) it.arrival = now_ns();
        items.push_back(it);
        Item& stored = items.back();
        if (submit(stored) != PARALLAX_OK) {
            stored.status = parallax_last_error();
            stored.done = now_ns();
            free_buf(stored);
        } else {
            std::lock_guard<std::mutex> g(mu);
            pending.push_back(items.size() - 1);
        }
        cv.notify_all();
        advance();
    }
    {
        std::lock_guard<std::mutex> g(mu);
        finished = true;
    }
    cv.notify_all();
    waiter.join();
}

void fill(void* p, int t, uint64_t seed) {
    const uint64_t n = kPoolElems;
    const int parts = 16;
    std::vector<std::thread> th;
    for (int k = 0; k < parts; ++k) {
        th.emplace_back([=] {
            const uint64_t a = n * k / parts, b = n * (k + 1) / parts;
            for (uint64_t i = a; i < b; ++i) {
                const uint64_t u = splitmix(seed * 0x9E3779B97F4A7C15ull + i);
                switch (t) {
                    case 0: static_cast<float*>(p)[i] = (float)((double)(u >> 40) * 0x1p-24); break;
                    case 1: static_cast<double*>(p)[i] = (double)(u >> 11) * 0x1p-53; break;
                    case 2: static_cast<int32_t*>(p)[i] = (int32_t)(u % 2001) - 1000; break;
                    default: static_cast<int64_t*>(p)[i] = (int64_t)u; break;
                }
            }
        });
    }
    for (auto& x : th) x.join();
}

}  // namespace

// Allocates and fills the shared inputs (once). Returns a parallax_status.
LG_EXPORT int px_loadgen_prepare(uint64_t seed) {
    if (g_pool.ready) return PARALLAX_OK;
    for (int t = 0; t < 4; ++t) {
        const size_t bytes = kPoolElems * kSize[t];
        g_pool.in[t] = parallax_arena_alloc(bytes, 256);
        if (!g_pool.in[t]) return PARALLAX_ERR_OUT_OF_MEMORY;
        fill(g_pool.in[t], t, seed + (uint64_t)t);
        int st = parallax_arena_set_residency(g_pool.in[t], PARALLAX_DEVICE_RESIDENT);
        if (st == PARALLAX_OK) st = parallax_arena_sync_to_device(g_pool.in[t], bytes);
        if (st != PARALLAX_OK) return st;
        char spec[64];
        snprintf(spec, sizeof spec, "reduce:sum:%s", kTypes[t]);
        g_pool.reduce[t] = parallax_builtin_kernel(spec);
        snprintf(spec, sizeof spec, "exclusive_scan:%s", kTypes[t]);
        g_pool.scan[t] = parallax_builtin_kernel(spec);
        snprintf(spec, sizeof spec, "sort:%s", kTypes[t]);
        g_pool.sort[t] = parallax_builtin_kernel(spec);
        snprintf(spec, sizeof spec, t < 2 ? "copy_if:%s:gt:0.5" : "copy_if:%s:gt:0", kTypes[t]);
        g_pool.copy_if[t] = parallax_builtin_kernel(spec);
        if (!g_pool.reduce[t] || !g_pool.scan[t] || !g_pool.sort[t] || !g_pool.copy_if[t])
            return PARALLAX_ERR_INVALID_HANDLE;
    }
    g_pool.ready = true;
    return PARALLAX_OK;
}

LG_EXPORT void px_loadgen_release(void) {
    for (int t = 0; t < 4; ++t) {
        if (g_pool.in[t]) parallax_arena_free(g_pool.in[t]);
        g_pool.in[t] = nullptr;
    }
    g_pool.ready = false;
}

// Runs one measurement; the serving loop must be running for modes 1 and 4.
LG_EXPORT int px_loadgen_run(const px_loadgen_config* cfg, px_loadgen_result* res) {
    if (!cfg || !res || !g_pool.ready) return PARALLAX_ERR_INVALID_ARGUMENT;
    px_loadgen_config c = *cfg;
    if (c.threads == 0) c.threads = 16;
    if (c.max_inflight == 0) c.max_inflight = 64;
    if (c.log2_max == 0) c.log2_max = 26;
    if (c.log2_min == 0) c.log2_min = 10;
    std::vector<ThreadOut> outs(c.threads);
    std::vector<std::thread> th;
    StartLine line;
    line.expected = c.threads;
    line.seconds = c.seconds;
    for (uint32_t i = 0; i < c.threads; ++i)
        th.emplace_back(client, std::cref(c), (int)i, &line, &outs[i]);
    for (auto& x : th) x.join();
    memset(res, 0, sizeof *res);
    std::vector<double> lat;
    uint64_t first = UINT64_MAX, last = 0;
    double bytes = 0;
    for (auto& o : outs)
        for (auto& it : o.items) {
            if (it.status != PARALLAX_OK) {
                ++res->errors;
                continue;
            }
            ++res->completed;
            ++res->per_op[it.op];
            lat.push_back((double)(it.done - it.arrival) * 1e-6);
            first = std::min(first, it.arrival);
            last = std::max(last, it.done);
            bytes += (double)alg_bytes(it);
        }
    if (lat.empty()) return PARALLAX_OK;
    std::sort(lat.begin(), lat.end());
    res->seconds = (double)(last - first) * 1e-9;
    res->req_s = res->completed / res->seconds;
    res->p50_ms = lat[lat.size() / 2];
    res->p99_ms = lat[std::min(lat.size() - 1, (size_t)(lat.size() * 0.99))];
    res->max_ms = lat.back();
    double sum = 0;
    for (double v : lat) sum += v;
    res->mean_ms = sum / lat.size();
    res->gbytes = bytes * 1e-9;
    res->gb_s = res->gbytes / res->seconds;
    return PARALLAX_OK;
}
