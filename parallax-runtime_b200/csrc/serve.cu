// Serving loop: continuous batching of primitive requests from many host threads.
//
// No reference counterpart: the reference runs one synchronous call at a time on a single
// command buffer and fence and is not thread-safe (src/kernel/kernel_launcher.hpp:172-176,
// src/kernel/kernel_launcher.cpp:438-443).
//
// Clients submit requests (reduce / scan / sort / copy_if over operands already resident on
// the device: PARALLAX_DEVICE_RESIDENT arena blocks or device memory) from any number of
// threads. `schedulers` host threads share the queued requests; each owns an equal share of
// `lanes` independent device lanes (a workspace each: stream, scratch, descriptor table,
// pinned result slots) and keeps them busy:
//   * completion: a lane whose batch finished (event query) hands every request its result
//     and releases the request's admitted bytes;
//   * admission: requests are taken in arrival order while the in-flight byte budget
//     allows (operands plus sort temporaries, which come from the lane's own buffer); the
//     head request that does not fit waits for completions (no overtaking, so no
//     starvation);
//   * coalescing: the head request and every queued request of the same kind (operation,
//     element type, predicate, scan flavour) up to `solo_elements` long become ONE
//     segmented launch over per-request descriptors (segmented.cu, sort.cu): a planner plus
//     one persistent kernel (every reduce, scan and compaction kind has one), or the
//     per-segment merge passes of the segmented sort. Longer requests and a request that
//     finds no partner run alone through the plain launchers.
// Requests that arrive while others are on the device are admitted into the next free
// lane, so batches overlap on the device; a request's result does not depend on what it
// was batched with (integer results are bit-exact, floating-point ones are within the
// primitives' stated tolerance of the fp64 oracle either way).
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include <atomic>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <chrono>
#include <thread>
#include <vector>

#include "runtime.hpp"
#include "segplan.cuh"

namespace pxb {
namespace {

enum class ReqOp : int { REDUCE, SCAN, SORT, COMPACT };

uint64_t now_ns() {
    timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (uint64_t)ts.tv_sec * 1000000000ull + (uint64_t)ts.tv_nsec;
}

struct Request {
    ReqOp op = ReqOp::REDUCE;
    DType t = DType::INVALID;  // U64 for sort_kv records
    bool by_key = false;       // sort_kv: records sorted stably by their high 32 bits
    RedOp red = RedOp::SUM;
    CompactMode mode = CompactMode::SELECT;
    Pred pred;                 // negate folded in (remove_if)
    bool exclusive = false;
    uint64_t init_bits = 0;
    const void* d_in = nullptr;
    void* d_out = nullptr;
    uint64_t n = 0;
    size_t es = 0;
    void* result = nullptr;    // caller's host memory: reduce value / kept count
    uint64_t footprint = 0;    // admitted bytes (operands + temporaries)
    bool coalescible = false;
    uint64_t seq = 0;          // arrival order
    // completion: the finisher writes status and done_ns, then sets `released` as its very
    // last access to the request; the waiter (which deletes the request afterwards) reads
    // them only once it sees `released`
    int status = PARALLAX_OK;
    uint64_t done_ns = 0;
    std::atomic<bool> released{false};
};

// No lock and no wake-up: a condition variable would make the scheduler thread issue a
// futex wake for every finished request whose waiter sleeps (measured: 4.3 us of scheduler
// time per small request, the serving loop's bound), so waiters poll the flag instead.
void finish(Request* r, int status) {
    r->status = status;
    r->done_ns = now_ns();
    r->released.store(true, std::memory_order_release);
}

// How long a waiter polls its request's flag before it sleeps (PARALLAX_SERVE_SPIN_US).
uint64_t spin_ns() {
    static const uint64_t ns = [] {
        const char* e = getenv("PARALLAX_SERVE_SPIN_US");
        return (e && *e ? strtoull(e, nullptr, 10) : 20ull) * 1000ull;
    }();
    return ns;
}

// Blocks until the request has been finished; returns its status. Short requests finish
// within microseconds of their launch, so the waiter first polls the completion flag (20 us
// by default), then sleeps between polls (about 20 us asked; the kernel's timer slack makes
// it longer), which costs a long request no more than that in latency.
int wait_request(Request* r, uint64_t* done_ns) {
    const uint64_t poll_until = now_ns() + spin_ns();
    for (int i = 1; !r->released.load(std::memory_order_acquire); ++i) {
        __builtin_ia32_pause();
        if ((i & 63) == 0 && now_ns() > poll_until) break;
    }
    while (!r->released.load(std::memory_order_acquire))
        std::this_thread::sleep_for(std::chrono::microseconds(20));
    if (done_ns) *done_ns = r->done_ns;
    return r->status;
}

// The kind of a coalescible request, as a map key: requests of equal keys run as one launch
// (operation, element type, sort_kv flavour, reduce operator, compaction mode, scan flavour
// and init, and the whole predicate: kind, negation, threshold, modulus and remainder).
struct KindKey {
    uint64_t v[8];
    bool operator<(const KindKey& o) const { return memcmp(v, o.v, sizeof v) < 0; }
};
KindKey kind_key(const Request& r) {
    KindKey k;
    memset(&k, 0, sizeof k);
    k.v[0] = (uint64_t)r.op | (uint64_t)(int)r.t << 8 | (uint64_t)r.by_key << 16 |
             (uint64_t)(int)r.red << 24 | (uint64_t)(int)r.mode << 32 | (uint64_t)r.exclusive << 40;
    k.v[1] = r.init_bits;
    k.v[2] = (uint64_t)(int)r.pred.kind | (uint64_t)r.pred.negate << 8;
    k.v[3] = (uint64_t)r.pred.i;
    k.v[4] = r.pred.u;
    double f = r.pred.f;
    if (f != f) f = __builtin_nan("");  // every NaN threshold is one kind
    memcpy(&k.v[5], &f, 8);
    k.v[6] = (uint64_t)r.pred.mod_m;
    k.v[7] = (uint64_t)r.pred.mod_r;
    return k;
}

struct Lane {
    Workspace* ws = nullptr;
    cudaEvent_t done = nullptr;
    SegDesc* h_desc = nullptr;   // pinned, mapped
    SegDesc* m_desc = nullptr;   // device alias of h_desc
    SegDesc* d_desc = nullptr;   // device
    uint64_t* h_res = nullptr;   // pinned, mapped: one 8-byte result slot per request
    uint64_t* d_res = nullptr;   // device alias of h_res
    std::vector<Request*> reqs;
    bool busy = false;
    // temporaries of a coalesced sort batch (one per request, 256-byte aligned): a
    // device-resident arena block, grown when a batch needs more (arena blocks come and go
    // without the device synchronisation of cudaMalloc / cudaFree, which would stall every
    // lane behind the running sorts); only this lane's scheduler thread touches it
    void* tmp_block = nullptr;  // host-side arena address
    size_t tmp_cap = 0;
};

class Server {
  public:
    parallax_serve_config cfg{};
    std::vector<Lane> lanes;
    std::vector<std::thread> thr;
    std::mutex mu;
    std::condition_variable cv_sched;
    // Queued requests: one FIFO per kind of coalescible request and one for requests that
    // run alone. Each request carries its arrival number, so the oldest queued request is the
    // oldest of the FIFO fronts, and a batch takes the head's kind from its FIFO directly
    // (no scan of the whole queue under the lock).
    std::map<KindKey, std::deque<Request*>> kinds;
    std::deque<Request*> solo;
    // queued is changed under mu; a scheduler reads it without mu to skip the lock when
    // there is nothing to form
    std::atomic<uint64_t> queued{0};
    uint64_t arrivals = 0;
    bool stopping = false;
    std::atomic<uint64_t> inflight{0};  // admitted bytes (released without the lock)
    parallax_serve_stats stats{};
    std::atomic<uint64_t> launch_ns{0}, complete_ns{0};  // scheduler time, all threads

    bool init(const parallax_serve_config* c) {
        if (c) cfg = *c;
        if (cfg.lanes == 0) cfg.lanes = 8;
        if (cfg.max_batch == 0) cfg.max_batch = 1024;
        if (cfg.solo_elements == 0) cfg.solo_elements = 1ull << 18;
        if (cfg.inflight_bytes == 0) cfg.inflight_bytes = parallax_arena_capacity() / 2;
        if (cfg.schedulers == 0) {
            const char* e = getenv("PARALLAX_SERVE_SCHEDULERS");
            cfg.schedulers = e && atoi(e) > 0 ? (uint32_t)atoi(e) : 2;
        }
        if (cfg.schedulers > cfg.lanes) cfg.schedulers = cfg.lanes;
        lanes.resize(cfg.lanes);
        for (Lane& l : lanes) {
            l.ws = new_workspace();
            if (!l.ws) return false;
            if (!cuda_ok(cudaEventCreateWithFlags(&l.done, cudaEventDisableTiming), "serve event") ||
                !cuda_ok(cudaHostAlloc((void**)&l.h_desc, cfg.max_batch * sizeof(SegDesc),
                                       cudaHostAllocMapped),
                         "serve descriptors (host)") ||
                !cuda_ok(cudaHostGetDevicePointer((void**)&l.m_desc, l.h_desc, 0),
                         "serve descriptors (host)") ||
                !cuda_ok(cudaMalloc((void**)&l.d_desc, cfg.max_batch * sizeof(SegDesc)),
                         "serve descriptors (device)") ||
                !cuda_ok(cudaHostAlloc((void**)&l.h_res, cfg.max_batch * 8, cudaHostAllocMapped),
                         "serve results") ||
                !cuda_ok(cudaHostGetDevicePointer((void**)&l.d_res, l.h_res, 0), "serve results"))
                return false;
        }
        // scheduler i owns lanes [i * L / N, (i + 1) * L / N); all take work from one queue
        for (uint32_t i = 0; i < cfg.schedulers; ++i) {
            const size_t lo = (size_t)i * lanes.size() / cfg.schedulers;
            const size_t hi = (size_t)(i + 1) * lanes.size() / cfg.schedulers;
            thr.emplace_back([this, lo, hi] { loop(lo, hi); });
        }
        return true;
    }

    void submit(Request* r) {
        r->coalescible = r->coalescible && r->n <= cfg.solo_elements;
        // a sort long enough for the radix path runs alone: the segmented sort merges
        if (r->op == ReqOp::SORT && r->n >= sort_radix_min(r->t)) r->coalescible = false;
        const KindKey key = r->coalescible ? kind_key(*r) : KindKey{};
        {
            std::lock_guard<std::mutex> g(mu);
            r->seq = arrivals++;
            (r->coalescible ? kinds[key] : solo).push_back(r);
            ++queued;
            ++stats.requests;
        }
        cv_sched.notify_one();
    }

    // Lane buffers go with the server (stop() has joined the threads; the lanes' workspaces
    // stay in the runtime's list, like every workspace).
    ~Server() {
        for (Lane& l : lanes) {
            if (l.ws) cudaStreamSynchronize(l.ws->stream());
            if (l.tmp_block) parallax_arena_free(l.tmp_block);
            if (l.d_desc) cudaFree(l.d_desc);
            if (l.h_desc) cudaFreeHost(l.h_desc);
            if (l.h_res) cudaFreeHost(l.h_res);
            if (l.done) cudaEventDestroy(l.done);
        }
        cudaGetLastError();
    }

    void stop() {
        {
            std::lock_guard<std::mutex> g(mu);
            stopping = true;
        }
        cv_sched.notify_all();
        for (std::thread& t : thr)
            if (t.joinable()) t.join();
    }

  private:
    // ---- admission (mutex held) ----------------------------------------------------------------
    // Admits r when the in-flight byte budget allows it (an idle server admits anything).
    bool admit(Request* r) {
        const uint64_t now = inflight.load();
        if (now != 0 && now + r->footprint > cfg.inflight_bytes) return false;
        const uint64_t after = inflight.fetch_add(r->footprint) + r->footprint;
        if (after > stats.peak_inflight_bytes) stats.peak_inflight_bytes = after;
        return true;
    }

    // Takes the next batch off the queues (mutex held); empty when the head must wait.
    std::vector<Request*> form_batch() {
        std::vector<Request*> b;
        if (!queued) return b;
        std::deque<Request*>* dq = solo.empty() ? nullptr : &solo;  // the oldest request's FIFO
        for (auto& kv : kinds)
            if (!kv.second.empty() && (!dq || kv.second.front()->seq < dq->front()->seq))
                dq = &kv.second;
        Request* head = dq->front();
        if (!admit(head)) {
            ++stats.memory_waits;
            return b;
        }
        dq->pop_front();
        --queued;
        b.push_back(head);
        if (head->coalescible) {  // its kind's later arrivals, in order
            while (!dq->empty() && b.size() < cfg.max_batch && admit(dq->front())) {
                b.push_back(dq->front());
                dq->pop_front();
                --queued;
            }
        }
        return b;
    }

    // ---- launch (no mutex) ---------------------------------------------------------------------
    bool launch(Lane& l) {
        Workspace& ws = *l.ws;
        const Request& h = *l.reqs[0];
        const size_t S = l.reqs.size();
        cudaStream_t s = ws.stream();
        if (!h.coalescible || S == 1) {  // one request: the plain launcher (fewer launches)
            l.h_res[0] = 0;
            switch (h.op) {
                case ReqOp::REDUCE: return launch_reduce(ws, h.t, h.red, h.d_in, h.n, l.d_res);
                case ReqOp::SCAN:
                    return launch_scan(ws, h.t, h.exclusive, h.d_in, h.d_out ? h.d_out : (void*)h.d_in,
                                       h.n, h.exclusive ? &h.init_bits : nullptr);
                case ReqOp::SORT:
                    return launch_sort(ws, h.t, const_cast<void*>(h.d_in), h.n, h.by_key);
                case ReqOp::COMPACT:
                    return launch_compact(ws, h.t, h.mode, h.pred, h.d_in, h.d_out, h.n, l.d_res);
            }
            return false;
        }
        char* tmp = nullptr;  // a sort batch's temporaries, from the lane's own buffer
        if (h.op == ReqOp::SORT) {
            size_t need = 0;
            for (size_t i = 0; i < S; ++i) need += (l.reqs[i]->n * l.reqs[i]->es + 255) / 256 * 256;
            if (need > l.tmp_cap) {  // the lane is idle between its batches: safe to replace
                if (l.tmp_block) parallax_arena_free(l.tmp_block);
                l.tmp_block = nullptr;
                l.tmp_cap = 0;
                const size_t cap = need + need / 2;
                void* blk = parallax_arena_alloc(cap, 256);
                if (!blk) {
                    set_error(PARALLAX_ERR_OUT_OF_MEMORY, "serve: sort temporaries of %zu bytes", need);
                    return false;
                }
                parallax_arena_set_residency(blk, PARALLAX_DEVICE_RESIDENT);
                l.tmp_block = blk;
                l.tmp_cap = cap;
            }
            tmp = static_cast<char*>(arena_dev(l.tmp_block));
        }
        uint64_t total = 0, max_len = 0;
        for (size_t i = 0; i < S; ++i) {
            const Request& r = *l.reqs[i];
            SegDesc& d = l.h_desc[i];
            l.h_res[i] = 0;
            d.in = reinterpret_cast<uint64_t>(r.d_in);
            d.out = reinterpret_cast<uint64_t>(r.d_out ? r.d_out : (void*)r.d_in);
            d.n = r.n;
            if (r.op == ReqOp::SORT) {
                d.aux = reinterpret_cast<uint64_t>(tmp);
                tmp += (r.n * r.es + 255) / 256 * 256;
            } else {
                d.aux = reinterpret_cast<uint64_t>(l.d_res + i);
            }
            total += r.n;
            if (r.n > max_len) max_len = r.n;
        }
        // Reduce, scan and compaction read the descriptors only in their planner (once per
        // segment and per work item), so they read the mapped host table in place: no
        // upload call. The sorts read them in every pass: they get a device copy.
        switch (h.op) {
            case ReqOp::REDUCE:
                return launch_segmented_descs(ws, SegKind::REDUCE, h.t, h.pred, false, 0, l.m_desc,
                                              S, total, h.red);
            case ReqOp::SCAN:
                return launch_segmented_descs(ws, SegKind::SCAN, h.t, h.pred, !h.exclusive,
                                              h.exclusive ? h.init_bits : 0, l.m_desc, S, total);
            case ReqOp::COMPACT:
                return launch_segmented_descs(ws, SegKind::COPY_IF, h.t, h.pred, false, 0, l.m_desc,
                                              S, total, RedOp::SUM, h.mode);
            case ReqOp::SORT:
                if (!cuda_ok(cudaMemcpyAsync(l.d_desc, l.h_desc, S * sizeof(SegDesc),
                                             cudaMemcpyHostToDevice, s),
                             "serve descriptor upload"))
                    return false;
                return launch_segmented_sort_descs(ws, h.t, l.d_desc, S, total, max_len, h.by_key);
        }
        return false;
    }

    // ---- completion (no mutex while reading results) ------------------------------------------------
    void complete(Lane& l, int status) {
        int32_t spin = l.ws->h_slot->spin_error;
        if (spin) {
            l.ws->h_slot->spin_error = 0;
            if (status == PARALLAX_OK) status = PARALLAX_ERR_DEVICE_SPIN;
        }
        for (size_t i = 0; i < l.reqs.size(); ++i) {
            Request* r = l.reqs[i];
            if (status == PARALLAX_OK && r->result) {
                const uint64_t v = l.h_res[l.reqs.size() > 1 ? i : 0];
                if (r->op == ReqOp::REDUCE) memcpy(r->result, &v, r->es);
                else if (r->op == ReqOp::COMPACT) memcpy(r->result, &v, 8);
            }
        }
        uint64_t released = 0;
        for (Request* r : l.reqs) released += r->footprint;
        inflight.fetch_sub(released);
        for (Request* r : l.reqs) finish(r, status);  // r may be deleted right after
        l.reqs.clear();
        l.busy = false;
    }

    void loop(size_t lo, size_t hi) {
        ensure_device();
        for (;;) {
            bool progress = false;
            bool any_busy = false;
            for (size_t li = lo; li < hi; ++li) {
                Lane& l = lanes[li];
                if (!l.busy) continue;
                const cudaError_t e = cudaEventQuery(l.done);
                if (e == cudaErrorNotReady) {
                    any_busy = true;
                    continue;
                }
                const uint64_t t0 = now_ns();
                complete(l, e == cudaSuccess ? PARALLAX_OK : PARALLAX_ERR_CUDA);
                complete_ns.fetch_add(now_ns() - t0, std::memory_order_relaxed);
                if (e != cudaSuccess) cudaGetLastError();
                progress = true;
            }
            if (any_busy && !progress) {
                // lanes still running: take the queue lock only when a request waits and one
                // of this scheduler's lanes is free (two schedulers polling their lanes would
                // otherwise hold the lock that every submission needs most of the time)
                bool free_lane = false;
                for (size_t li = lo; li < hi && !free_lane; ++li) free_lane = !lanes[li].busy;
                if (!free_lane || queued.load(std::memory_order_relaxed) == 0) {
                    std::this_thread::yield();
                    continue;
                }
            }
            std::unique_lock<std::mutex> lk(mu);
            for (size_t li = lo; li < hi; ++li) {
                Lane& l = lanes[li];
                if (l.busy || !queued) continue;
                const uint64_t t0 = now_ns();
                std::vector<Request*> b = form_batch();
                if (b.empty()) break;
                l.reqs = std::move(b);
                l.busy = true;
                ++stats.batches;
                if (l.reqs.size() > stats.max_batch) stats.max_batch = l.reqs.size();
                if (l.reqs.size() > 1) stats.coalesced_requests += l.reqs.size();
                else ++stats.solo_batches;
                lk.unlock();
                set_ok();
                const bool ok = launch(l) &&
                                cuda_ok(cudaEventRecord(l.done, l.ws->stream()), "serve event record");
                if (!ok) {
                    // drain what the failed launch enqueued before its buffers are reused
                    const int st = last_error() ? last_error() : PARALLAX_ERR_CUDA;
                    cudaStreamSynchronize(l.ws->stream());
                    cudaGetLastError();
                    complete(l, st);
                }
                launch_ns.fetch_add(now_ns() - t0, std::memory_order_relaxed);
                lk.lock();
                progress = true;
                any_busy = true;
            }
            if (stopping && !queued && !any_busy) {
                bool busy = false;
                for (size_t li = lo; li < hi; ++li) busy |= lanes[li].busy;
                if (!busy) break;
            }
            if (progress) continue;
            if (any_busy) {
                lk.unlock();
                std::this_thread::yield();  // poll the lanes' events
            } else {
                cv_sched.wait(lk, [&] { return stopping || queued; });
            }
        }
    }
};

std::mutex g_srv_mu;
Server* g_srv = nullptr;

// Builds a request from the public description; returns a parallax_status.
int make_request(const parallax_request* q, Request* r) {
    static const char* fn = "parallax_serve_submit";
    Handle* h = q ? as_handle(q->kernel) : nullptr;
    if (!h) {
        set_error(PARALLAX_ERR_INVALID_HANDLE, "%s: invalid kernel handle", fn);
        return PARALLAX_ERR_INVALID_HANDLE;
    }
    r->t = h->kind == Kind::SORT_KV ? DType::U64 : h->dtype;
    r->es = dtype_size(r->t);
    r->n = q->count;
    r->result = q->result;
    switch (h->kind) {
        case Kind::REDUCE:
            r->op = ReqOp::REDUCE;
            r->red = h->op;
            r->coalescible = true;
            break;
        case Kind::SCAN:
            r->op = ReqOp::SCAN;
            r->exclusive = (q->flags & PARALLAX_REQ_EXCLUSIVE) != 0;
            if (r->exclusive && q->init) memcpy(&r->init_bits, q->init, r->es);
            r->coalescible = true;
            break;
        case Kind::SORT:
        case Kind::SORT_KV:
            r->op = ReqOp::SORT;
            r->by_key = h->kind == Kind::SORT_KV;
            r->coalescible = true;
            break;
        case Kind::COMPACT_FLAGS:
        case Kind::UNIQUE_FLAGS:
        case Kind::PARTITION_SCATTER:
            r->op = ReqOp::COMPACT;
            r->pred = h->pred;
            if (h->kind == Kind::COMPACT_FLAGS && h->remove) r->pred.negate = !r->pred.negate;
            r->mode = h->kind == Kind::UNIQUE_FLAGS ? CompactMode::UNIQUE
                    : h->kind == Kind::PARTITION_SCATTER ? CompactMode::PARTITION
                                                         : CompactMode::SELECT;
            r->coalescible = true;
            break;
        default:
            set_error(PARALLAX_ERR_INVALID_HANDLE, "%s: no served form for this kernel", fn);
            return PARALLAX_ERR_INVALID_HANDLE;
    }
    if (r->n == 0) return PARALLAX_OK;
    if (!(r->d_in = device_operand(q->input, fn, "input"))) return last_error();
    const bool has_out = r->op == ReqOp::COMPACT || (r->op == ReqOp::SCAN && q->output);
    if (has_out && !(r->d_out = device_operand(q->output, fn, "output"))) return last_error();
    r->footprint = r->n * r->es * (has_out ? 2 : 1) + (r->op == ReqOp::SORT ? r->n * r->es : 0);
    return PARALLAX_OK;
}

}  // namespace
}  // namespace pxb

using namespace pxb;

PXB_EXPORT int parallax_serve_start(const parallax_serve_config* cfg) {
    set_ok();
    if (!ensure_device()) {
        set_error(PARALLAX_ERR_NO_DEVICE, "no CUDA device available");
        return PARALLAX_ERR_NO_DEVICE;
    }
    std::lock_guard<std::mutex> g(g_srv_mu);
    if (g_srv) return PARALLAX_OK;
    auto* s = new Server();
    if (!s->init(cfg)) {
        delete s;  // lanes' workspaces stay in the global list (never freed by design)
        return last_error() ? last_error() : PARALLAX_ERR_CUDA;
    }
    g_srv = s;
    return PARALLAX_OK;
}

PXB_EXPORT int parallax_serve_stop(void) {
    Server* s;
    {
        std::lock_guard<std::mutex> g(g_srv_mu);
        s = g_srv;
        g_srv = nullptr;
    }
    if (!s) return PARALLAX_OK;
    s->stop();
    delete s;
    return PARALLAX_OK;
}

PXB_EXPORT int parallax_serve_submit(const parallax_request* req, uint64_t* ticket) {
    settle_deferred_here();  // a transform held back on this thread may produce the operand
    set_ok();
    if (!ticket) {
        set_error(PARALLAX_ERR_INVALID_ARGUMENT, "parallax_serve_submit: ticket is null");
        return PARALLAX_ERR_INVALID_ARGUMENT;
    }
    *ticket = 0;
    Server* s;
    {
        std::lock_guard<std::mutex> g(g_srv_mu);
        s = g_srv;
    }
    if (!s) {
        set_error(PARALLAX_ERR_SHUTDOWN, "parallax_serve_submit: the serving loop is not running");
        return PARALLAX_ERR_SHUTDOWN;
    }
    auto* r = new Request();
    const int st = make_request(req, r);
    if (st != PARALLAX_OK) {
        delete r;
        return st;
    }
    if (r->n == 0) {  // nothing to do on the device
        if (r->result && (r->op == ReqOp::REDUCE || r->op == ReqOp::COMPACT))
            memset(r->result, 0, r->op == ReqOp::REDUCE ? r->es : 8);
        finish(r, PARALLAX_OK);
    } else {
        s->submit(r);
    }
    *ticket = reinterpret_cast<uint64_t>(r);
    return PARALLAX_OK;
}

PXB_EXPORT int parallax_serve_wait(uint64_t ticket, uint64_t* done_ns) {
    set_ok();
    auto* r = reinterpret_cast<Request*>(ticket);
    if (!r) {
        set_error(PARALLAX_ERR_INVALID_ARGUMENT, "parallax_serve_wait: null ticket");
        return PARALLAX_ERR_INVALID_ARGUMENT;
    }
    // The request carries its own completion state, so waiting needs no server: a request
    // submitted before parallax_serve_stop() has been finished by the time stop returns
    // (stop drains the queue), and its status is returned here as usual.
    int st;
    if (r->n == 0) {  // finished at submission by this thread
        st = r->status;
        if (done_ns) *done_ns = r->done_ns;
    } else {
        st = wait_request(r, done_ns);
    }
    delete r;
    if (st != PARALLAX_OK) set_error(st, "served request failed (status %d)", st);
    return st;
}

PXB_EXPORT int parallax_serve_poll(uint64_t ticket, int* finished, uint64_t* done_ns) {
    set_ok();
    auto* r = reinterpret_cast<Request*>(ticket);
    if (!r || !finished) {
        set_error(PARALLAX_ERR_INVALID_ARGUMENT, "parallax_serve_poll: null ticket or flag");
        return PARALLAX_ERR_INVALID_ARGUMENT;
    }
    // One acquire load: a client that keeps many requests in flight checks its oldest one
    // between submissions, with no thread of its own blocked in parallax_serve_wait.
    if (!r->released.load(std::memory_order_acquire)) {
        *finished = 0;
        return PARALLAX_OK;
    }
    *finished = 1;
    const int st = r->status;
    if (done_ns) *done_ns = r->done_ns;
    delete r;
    if (st != PARALLAX_OK) set_error(st, "served request failed (status %d)", st);
    return st;
}

PXB_EXPORT int parallax_serve_call(const parallax_request* req) {
    uint64_t t = 0;
    const int st = parallax_serve_submit(req, &t);
    if (st != PARALLAX_OK) return st;
    return parallax_serve_wait(t, nullptr);
}

PXB_EXPORT int parallax_serve_get_stats(parallax_serve_stats* out) {
    if (!out) return PARALLAX_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> g(g_srv_mu);
    if (!g_srv) {
        memset(out, 0, sizeof *out);
        return PARALLAX_ERR_SHUTDOWN;
    }
    std::lock_guard<std::mutex> g2(g_srv->mu);
    *out = g_srv->stats;
    out->launch_ns = g_srv->launch_ns.load();
    out->complete_ns = g_srv->complete_ns.load();
    out->inflight_bytes = g_srv->inflight.load();
    out->queued = g_srv->queued;
    return PARALLAX_OK;
}

PXB_EXPORT uint64_t parallax_clock_ns(void) { return now_ns(); }
