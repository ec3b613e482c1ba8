// Device context, per-thread workspaces, error reporting and bounded host waits.
//
// Replaces the reference's Vulkan backend + single command buffer/fence
// (src/backend/vulkan/device.cpp:14-43, src/kernel/kernel_launcher.cpp:54-100,
// :438-443): one CUDA device, one non-blocking stream per submitting host thread, and
// host waits that poll an event against a deadline instead of waiting forever.
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include <unistd.h>

#include <algorithm>
#include <chrono>
#include <mutex>
#include <thread>
#include <vector>

#include "lookback.cuh"
#include "runtime.hpp"

namespace pxb {

// ---- errors ------------------------------------------------------------------------------
static thread_local int tls_status = 0;

static bool debug_enabled() {
    static const bool on = getenv("PARALLAX_DEBUG") != nullptr;
    return on;
}

void set_error(int status, const char* fmt, ...) {
    tls_status = status;
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    fprintf(stderr, "[parallax] %s\n", buf);
}
void set_ok() { tls_status = 0; }
int last_error() { return tls_status; }

bool cuda_ok(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return true;
    set_error(PARALLAX_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
    return false;
}

// ---- device ------------------------------------------------------------------------------
static DeviceInfo g_dev;
static std::once_flag g_dev_once;
static bool g_dev_ok = false;
static std::atomic<uint64_t> g_launches{0};

bool ensure_device() {
    std::call_once(g_dev_once, [] {
        int n = 0;
        if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
            cudaGetLastError();
            return;
        }
        int dev = 0;
        if (const char* e = getenv("PARALLAX_DEVICE")) dev = atoi(e);
        if (dev < 0 || dev >= n) dev = 0;
        if (cudaSetDevice(dev) != cudaSuccess) return;
        cudaDeviceProp prop;
        if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) return;
        g_dev.device = dev;
        g_dev.sm_count = prop.multiProcessorCount;
        g_dev.max_threads_per_sm = prop.maxThreadsPerMultiProcessor;
        g_dev.smem_per_sm = prop.sharedMemPerMultiprocessor;
        snprintf(g_dev.name, sizeof g_dev.name, "%s", prop.name);
        g_dev_ok = true;
        if (debug_enabled())
            fprintf(stderr, "[parallax] device %d: %s, %d SMs, cc %d.%d\n", dev, prop.name,
                    prop.multiProcessorCount, prop.major, prop.minor);
    });
    if (g_dev_ok) cudaSetDevice(g_dev.device);  // per-thread current device
    return g_dev_ok;
}
const DeviceInfo& device_info() { return g_dev; }
void count_launch(unsigned n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
uint64_t launch_count() { return g_launches.load(std::memory_order_relaxed); }

// ---- workspaces ------------------------------------------------------------------------------
// Workspaces are owned by a global list and never destroyed before process exit: a
// thread that exits leaves its (idle) stream and scratch behind, which keeps teardown
// order trivial for a library loaded into arbitrary host programs.
static std::mutex g_ws_mu;
static std::vector<Workspace*>* g_ws_list = nullptr;
static thread_local Workspace* tls_ws = nullptr;

Workspace* current_workspace() { return tls_ws; }

Workspace* workspace() {
    if (tls_ws) return tls_ws;
    tls_ws = new_workspace();
    return tls_ws;
}

Workspace* new_workspace() {
    if (!ensure_device()) {
        set_error(PARALLAX_ERR_NO_DEVICE, "no CUDA device available");
        return nullptr;
    }
    auto* ws = new Workspace();
    if (!cuda_ok(cudaStreamCreateWithFlags(&ws->own_stream, cudaStreamNonBlocking),
                 "cudaStreamCreate") ||
        !cuda_ok(cudaHostAlloc((void**)&ws->h_slot, sizeof(HostSlot), cudaHostAllocMapped),
                 "cudaHostAlloc(slot)") ||
        !cuda_ok(cudaHostGetDevicePointer((void**)&ws->d_slot, ws->h_slot, 0),
                 "cudaHostGetDevicePointer") ||
        !cuda_ok(cudaEventCreateWithFlags(&ws->done, cudaEventDisableTiming),
                 "cudaEventCreate")) {
        delete ws;
        return nullptr;
    }
    memset(ws->h_slot, 0, sizeof(HostSlot));
    {
        std::lock_guard<std::mutex> g(g_ws_mu);
        if (!g_ws_list) g_ws_list = new std::vector<Workspace*>();
        g_ws_list->push_back(ws);
    }
    return ws;
}

// Bytes of one look-back status entry (lookback.cuh): {u32 flag, u32 pad, u64 agg,
// u64 inc} for every accumulator type, so flag words sit at the same addresses in every
// launch.
static constexpr size_t kStatusEntry = sizeof(StatusEntry);

// Replaces a workspace buffer by a larger one (at least `bytes`, doubling from `min_cap`),
// optionally zeroed. In stream order: cudaFreeAsync / cudaMallocAsync on the workspace's
// stream wait only for that stream's earlier work (which may still use the old buffer),
// where cudaStreamSynchronize + cudaFree + cudaMalloc would also wait for every other stream
// of the device - a lane of the serving loop that met a larger request than before stalled
// behind the other lanes' running sorts. Growth inside a stream capture is refused.
static bool regrow(Workspace& ws, void** buf, size_t* cap_io, size_t bytes, size_t min_cap,
                   bool zero, const char* what) {
    cudaStream_t s = ws.stream();
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone) {
        set_error(PARALLAX_ERR_INVALID_ARGUMENT, "%s: buffer growth inside a stream capture", what);
        return false;
    }
    cudaGetLastError();
    if (*buf) {
        if (!cuda_ok(cudaFreeAsync(*buf, s), what)) return false;
        *buf = nullptr;
        *cap_io = 0;
    }
    size_t cap = min_cap;
    while (cap < bytes) cap <<= 1;
    if (!cuda_ok(cudaMallocAsync(buf, cap, s), what)) {
        *buf = nullptr;
        return false;
    }
    if (zero && !cuda_ok(cudaMemsetAsync(*buf, 0, cap, s), what)) return false;
    *cap_io = cap;
    ++ws.generation;
    return true;
}

char* Workspace::scratch(uint64_t tiles) {
    size_t bytes = kScratchSmall + tiles * kStatusEntry;
    if (bytes <= scratch_cap) return static_cast<char*>(d_scratch);
    // Zeroed: look-back status words then read as "not ready" for every epoch, and the
    // self-resetting ticket counters start at zero.
    if (!regrow(*this, &d_scratch, &scratch_cap, bytes, 1 << 20, true, "scratch")) return nullptr;
    epoch = 1;
    return static_cast<char*>(d_scratch);
}

void* Workspace::seg(size_t bytes) {
    if (bytes <= seg_cap) return d_seg;
    return regrow(*this, &d_seg, &seg_cap, bytes, 1 << 20, true, "segment buffer") ? d_seg : nullptr;
}

void* Workspace::seg_status(uint64_t entries) {
    if (entries <= seg_status_cap) return d_seg_status;
    size_t bytes_cap = seg_status_cap * kStatusEntry;
    if (!regrow(*this, &d_seg_status, &bytes_cap, entries * kStatusEntry, (1 << 14) * kStatusEntry,
                true, "segment status"))
        return nullptr;
    seg_status_cap = bytes_cap / kStatusEntry;
    return d_seg_status;
}

void* Workspace::radix(size_t bytes) {
    if (bytes <= radix_cap) return d_radix;
    if (!regrow(*this, &d_radix, &radix_cap, bytes, 1 << 20, true, "radix buffer")) return nullptr;
    radix_epoch = 1;
    return d_radix;
}

void* Workspace::seg_radix(size_t bytes) {
    if (bytes <= seg_radix_cap) return d_seg_radix;
    return regrow(*this, &d_seg_radix, &seg_radix_cap, bytes, 1 << 20, true,
                  "segmented radix buffer")
               ? d_seg_radix
               : nullptr;
}

bool Workspace::copy_streams() {
    if (copy_up && copy_down && ev_copy[3]) return true;
    if (!copy_up && !cuda_ok(cudaStreamCreateWithFlags(&copy_up, cudaStreamNonBlocking),
                             "cudaStreamCreate(upload)"))
        return false;
    if (!copy_down && !cuda_ok(cudaStreamCreateWithFlags(&copy_down, cudaStreamNonBlocking),
                               "cudaStreamCreate(download)"))
        return false;
    for (cudaEvent_t& e : ev_copy)
        if (!e && !cuda_ok(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate"))
            return false;
    return true;
}

uint32_t Workspace::next_radix_epochs(uint32_t count) {
    if (radix_epoch + count >= (1u << 22)) {
        cudaMemsetAsync(d_radix, 0, radix_cap, stream());
        radix_epoch = 1;
    }
    const uint32_t e = radix_epoch;
    radix_epoch += count;
    return e;
}

bool graph_launch(Workspace& ws, const std::string& key, const std::function<bool()>& enqueue) {
    static const bool enabled =
        !(getenv("PARALLAX_GRAPHS") && atoi(getenv("PARALLAX_GRAPHS")) == 0);
    if (!enabled) return enqueue();
    cudaStream_t s = ws.stream();
    if (ws.user_stream) {  // the caller may be capturing its own stream: launch into that
        cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
        if (cudaStreamIsCapturing(s, &st) != cudaSuccess || st != cudaStreamCaptureStatusNone) {
            cudaGetLastError();
            return enqueue();
        }
    }
    auto it = ws.graphs.find(key);
    if (it != ws.graphs.end() && it->second.first != ws.generation) {
        cudaGraphExecDestroy(it->second.second);
        ws.graphs.erase(it);
        it = ws.graphs.end();
    }
    if (it == ws.graphs.end()) {
        const uint64_t gen = ws.generation;
        cudaGraph_t g = nullptr;
        if (!cuda_ok(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "begin capture"))
            return false;
        const bool ok = enqueue();
        cudaError_t e = cudaStreamEndCapture(s, &g);
        if (!ok || !cuda_ok(e, "end capture")) {
            if (g) cudaGraphDestroy(g);
            return false;
        }
        if (ws.generation != gen) {  // a buffer moved during capture: cannot cache this graph
            cudaGraphDestroy(g);
            set_error(PARALLAX_ERR_CUDA, "workspace buffer reallocated during graph capture");
            return false;
        }
        cudaGraphExec_t exec = nullptr;
        e = cudaGraphInstantiate(&exec, g, 0);
        cudaGraphDestroy(g);
        if (!cuda_ok(e, "graph instantiate")) return false;
        it = ws.graphs.emplace(key, std::make_pair(gen, exec)).first;
    }
    return cuda_ok(cudaGraphLaunch(it->second.second, s), "graph launch");
}

void* Workspace::temp(size_t bytes) {
    if (bytes <= temp_cap) return d_temp;
    return regrow(*this, &d_temp, &temp_cap, bytes, 1 << 20, false, "temp") ? d_temp : nullptr;
}

void* Workspace::stage(int slot, size_t bytes) {
    if (bytes <= stage_cap[slot]) return d_stage[slot];
    return regrow(*this, &d_stage[slot], &stage_cap[slot], bytes, 1 << 20, false, "stage")
               ? d_stage[slot]
               : nullptr;
}

uint32_t Workspace::next_epoch() {
    // 30 bits of epoch sit above a 2-bit state in each status word. On wrap-around the
    // scratch is cleared so no stale word can alias a reused epoch.
    uint32_t e = epoch++;
    if (epoch >= (1u << 30)) {
        cudaMemsetAsync(d_scratch, 0, scratch_cap, stream());
        epoch = 1;
        e = epoch++;
    }
    return e;
}

// ---- profiling -------------------------------------------------------------------------------
namespace {
struct ProfRecord {
    const char* name;
    uint64_t bytes;
    cudaEvent_t start, stop;
};
std::atomic<bool> g_prof_on{false};
std::mutex g_prof_mu;
std::vector<ProfRecord>* g_prof = nullptr;
std::vector<cudaEvent_t>* g_event_pool = nullptr;

cudaEvent_t take_event() {
    std::lock_guard<std::mutex> g(g_prof_mu);
    if (!g_event_pool) g_event_pool = new std::vector<cudaEvent_t>();
    if (!g_event_pool->empty()) {
        cudaEvent_t e = g_event_pool->back();
        g_event_pool->pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}
}  // namespace

ProfScope::ProfScope(Workspace& ws, const char* kernel, uint64_t alg_bytes) {
    if (!g_prof_on.load(std::memory_order_relaxed)) return;
    ws_ = &ws;
    name_ = kernel;
    bytes_ = alg_bytes;
    start_ = take_event();
    cudaEventRecord(start_, ws.stream());
}
ProfScope::~ProfScope() {
    if (!ws_) return;
    cudaEvent_t stop = take_event();
    cudaEventRecord(stop, ws_->stream());
    std::lock_guard<std::mutex> g(g_prof_mu);
    if (!g_prof) g_prof = new std::vector<ProfRecord>();
    g_prof->push_back({name_, bytes_, start_, stop});
}

uint32_t wait_limit() {
    static const uint32_t v = [] {
        const char* e = getenv("PARALLAX_WAIT_LIMIT");
        const long long t = e ? atoll(e) : 0;
        return t > 0 && t < (long long)kSpinLimit ? (uint32_t)t : kSpinLimit;
    }();
    return v;
}

static long sync_timeout_ms() {
    static const long v = [] {
        const char* e = getenv("PARALLAX_SYNC_TIMEOUT_MS");
        long t = e ? atol(e) : 120000;
        return t > 0 ? t : 120000;
    }();
    return v;
}

int sync_stream(Workspace& ws) {
    cudaStream_t s = ws.stream();
    if (!cuda_ok(cudaEventRecord(ws.done, s), "cudaEventRecord")) return PARALLAX_ERR_CUDA;
    auto t0 = std::chrono::steady_clock::now();
    const long limit = sync_timeout_ms();
    unsigned spins = 0;
    for (;;) {
        cudaError_t q = cudaEventQuery(ws.done);
        if (q == cudaSuccess) break;
        if (q != cudaErrorNotReady) {
            cuda_ok(q, "kernel execution");
            return PARALLAX_ERR_CUDA;
        }
        // Spin briefly for low latency, then back off to avoid burning a core.
        if (++spins > 2000) {
            std::this_thread::sleep_for(std::chrono::microseconds(spins > 20000 ? 200 : 20));
            auto ms = std::chrono::duration_cast<std::chrono::milliseconds>(
                          std::chrono::steady_clock::now() - t0)
                          .count();
            if (ms > limit) {
                set_error(PARALLAX_ERR_TIMEOUT, "device work did not finish within %ld ms",
                          limit);
                return PARALLAX_ERR_TIMEOUT;
            }
        }
    }
    if (ws.h_slot->spin_error) {
        int code = ws.h_slot->spin_error;
        ws.h_slot->spin_error = 0;
        if (code == kErrMergeSpan) {
            set_error(PARALLAX_ERR_CUDA, "sort: a merge pass met an unsorted run (tile skipped)");
            return PARALLAX_ERR_CUDA;
        }
        if (code == kErrRadixRange) {
            set_error(PARALLAX_ERR_CUDA, "sort: a radix pass met an out-of-range position (skipped)");
            return PARALLAX_ERR_CUDA;
        }
        if (code == kErrSegmentOffsets) {
            set_error(PARALLAX_ERR_INVALID_ARGUMENT,
                      "segment offsets must be non-decreasing and within [0, count]");
            return PARALLAX_ERR_INVALID_ARGUMENT;
        }
        set_error(PARALLAX_ERR_DEVICE_SPIN, "an in-kernel bounded wait gave up (code %d)", code);
        return PARALLAX_ERR_DEVICE_SPIN;
    }
    return PARALLAX_OK;
}

}  // namespace pxb

// ---- exported: errors / streams / instrumentation ---------------------------------------------
using namespace pxb;

PXB_EXPORT int parallax_last_error(void) { return last_error(); }
PXB_EXPORT void parallax_clear_error(void) { set_ok(); }
PXB_EXPORT const char* parallax_error_string(int status) {
    switch (status) {
        case PARALLAX_OK: return "ok";
        case PARALLAX_ERR_INVALID_HANDLE: return "invalid kernel handle";
        case PARALLAX_ERR_INVALID_ARGUMENT: return "invalid argument";
        case PARALLAX_ERR_OUT_OF_MEMORY: return "out of memory";
        case PARALLAX_ERR_CUDA: return "CUDA error";
        case PARALLAX_ERR_TIMEOUT: return "host wait deadline passed";
        case PARALLAX_ERR_DEVICE_SPIN: return "in-kernel bounded wait gave up";
        case PARALLAX_ERR_UNSUPPORTED: return "unsupported";
        case PARALLAX_ERR_NO_DEVICE: return "no CUDA device";
        case PARALLAX_ERR_SHUTDOWN: return "runtime shut down";
        default: return "unknown status";
    }
}

PXB_EXPORT int parallax_set_stream(void* cuda_stream) {
    settle_deferred_here();
    Workspace* ws = workspace();
    if (!ws) return PARALLAX_ERR_NO_DEVICE;
    cudaStream_t next = static_cast<cudaStream_t>(cuda_stream);
    cudaStream_t prev = ws->stream();
    if ((next ? next : ws->own_stream) != prev) {
        // The workspace buffers pass from one stream to the other: work on the new stream
        // is ordered after what the old one has enqueued (async calls still running there
        // use the same scratch, and buffer growth frees in stream order).
        if (!cuda_ok(cudaEventRecord(ws->done, prev), "cudaEventRecord(set_stream)") ||
            !cuda_ok(cudaStreamWaitEvent(next ? next : ws->own_stream, ws->done, 0),
                     "cudaStreamWaitEvent(set_stream)"))
            return PARALLAX_ERR_CUDA;
    }
    ws->user_stream = next;
    return PARALLAX_OK;
}
PXB_EXPORT int parallax_set_async(int async) {
    settle_deferred_here();
    Workspace* ws = workspace();
    if (!ws) return PARALLAX_ERR_NO_DEVICE;
    ws->async = async != 0;
    return PARALLAX_OK;
}
PXB_EXPORT int parallax_synchronize(void) {
    settle_deferred_here();
    Workspace* ws = workspace();
    if (!ws) return PARALLAX_ERR_NO_DEVICE;
    int st = sync_stream(*ws);
    if (st == PARALLAX_OK) ws->last_count = ws->h_slot->count[0];
    return st;
}
PXB_EXPORT size_t parallax_last_count(void) {
    Workspace* ws = workspace();
    return ws ? ws->last_count : 0;
}
PXB_EXPORT uint64_t parallax_launch_count(void) { return launch_count(); }

PXB_EXPORT void parallax_profile_enable(int on) { g_prof_on.store(on != 0); }

namespace {
struct ProfAgg {
    uint64_t launches = 0, bytes = 0;
    double ms = 0;
};
std::vector<std::pair<std::string, ProfAgg>> g_prof_aggs;  // guarded by g_prof_agg_mu
std::mutex g_prof_agg_mu;
}  // namespace

PXB_EXPORT void parallax_profile_reset(void) {
    std::lock_guard<std::mutex> g(g_prof_agg_mu);
    g_prof_aggs.clear();
}

// Folds the launches recorded so far (waiting for them to finish) into per-kernel totals
// and writes {"kernel": {"launches": L, "ms": T, "alg_bytes": B}, ...} into buf. Returns
// the length the full JSON needs (excluding the terminator). Totals accumulate until
// parallax_profile_reset().
PXB_EXPORT size_t parallax_profile_json(char* buf, size_t cap) {
    std::vector<ProfRecord> recs;
    {
        std::lock_guard<std::mutex> g(g_prof_mu);
        if (g_prof) recs.swap(*g_prof);
    }
    std::lock_guard<std::mutex> ga(g_prof_agg_mu);
    auto& aggs = g_prof_aggs;
    for (auto& r : recs) {
        cudaEventSynchronize(r.stop);
        float ms = 0;
        cudaEventElapsedTime(&ms, r.start, r.stop);
        auto it = std::find_if(aggs.begin(), aggs.end(),
                               [&](const auto& a) { return a.first == r.name; });
        if (it == aggs.end()) {
            aggs.emplace_back(r.name, ProfAgg{});
            it = aggs.end() - 1;
        }
        it->second.launches++;
        it->second.bytes += r.bytes;
        it->second.ms += ms;
    }
    {
        std::lock_guard<std::mutex> g(g_prof_mu);
        if (!g_event_pool) g_event_pool = new std::vector<cudaEvent_t>();
        for (auto& r : recs) {
            g_event_pool->push_back(r.start);
            g_event_pool->push_back(r.stop);
        }
    }
    std::string out = "{";
    char tmp[256];
    for (size_t i = 0; i < aggs.size(); ++i) {
        snprintf(tmp, sizeof tmp, "%s\"%s\": {\"launches\": %llu, \"ms\": %.6f, \"alg_bytes\": %llu}",
                 i ? ", " : "", aggs[i].first.c_str(), (unsigned long long)aggs[i].second.launches,
                 aggs[i].second.ms, (unsigned long long)aggs[i].second.bytes);
        out += tmp;
    }
    out += "}";
    if (buf && cap) snprintf(buf, cap, "%s", out.c_str());
    return out.size();
}
PXB_EXPORT int parallax_device_info(int* device, int* sm_count, char* name, size_t name_cap) {
    if (!ensure_device()) return PARALLAX_ERR_NO_DEVICE;
    if (device) *device = g_dev.device;
    if (sm_count) *sm_count = g_dev.sm_count;
    if (name && name_cap) snprintf(name, name_cap, "%s", g_dev.name);
    return PARALLAX_OK;
}
