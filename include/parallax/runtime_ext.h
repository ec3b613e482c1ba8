/*
 * Additive entry points of the B200 parallax runtime. None of these exists in the
 * reference ABI; code that links only against parallax/runtime.h never needs them.
 * They expose what the reference's synchronous, host-coherent ABI cannot express:
 * device residency of arena blocks, stream-ordered (asynchronous) calls, built-in
 * kernel handles without a compiler, segmented launches and the serving loop.
 */
#ifndef PARALLAX_RUNTIME_EXT_H
#define PARALLAX_RUNTIME_EXT_H

#include <stddef.h>
#include <stdint.h>
#include "parallax/runtime.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---- errors ---------------------------------------------------------------------- */
enum parallax_status {
    PARALLAX_OK = 0,
    PARALLAX_ERR_INVALID_HANDLE = 1,
    PARALLAX_ERR_INVALID_ARGUMENT = 2,
    PARALLAX_ERR_OUT_OF_MEMORY = 3,
    PARALLAX_ERR_CUDA = 4,
    PARALLAX_ERR_TIMEOUT = 5,        /* a host wait passed its deadline */
    PARALLAX_ERR_DEVICE_SPIN = 6,    /* an in-kernel bounded wait gave up */
    PARALLAX_ERR_UNSUPPORTED = 7,
    PARALLAX_ERR_NO_DEVICE = 8,
    PARALLAX_ERR_SHUTDOWN = 9,
};
/* Status of the calling thread's most recent ABI call. */
int parallax_last_error(void);
const char* parallax_error_string(int status);
void parallax_clear_error(void);

/* ---- built-in kernels ------------------------------------------------------------ */
/* Handle for a built-in sm_100a kernel named by a spec string:
 *   "reduce:<sum|max|min>:<dtype>"        "scan:<dtype>"   "exclusive_scan:<dtype>"
 *   "sort:<dtype>"                        "sort_kv:u32"   (u64 composite (key<<32|value))
 *   "copy_if:<dtype>:<pred>"              "remove_if:<dtype>:<pred>"
 *   "partition:<dtype>:<pred>"            "unique:<dtype>"
 *   "count_if:<dtype>:<pred>"             "find:<dtype>:<pred>"
 *   "argminmax:<dtype>"                   "mismatch:<dtype>"
 *   "map:<name>"                          fixed element-wise ops: "map:saxpy_gather_f32"
 *                                         (transform2 of 16-byte {float x; u32 pad;
 *                                         float* p} records to y = a*x + *p, a = the
 *                                         first 4 capture bytes), "map:affine_f32"
 *                                         (in-place x = a*x + b, captures {a, b})
 * dtype: f32 f64 i32 i64 u32 u64. pred: gt:<c> ge:<c> lt:<c> le:<c> eq:<c> ne:<c>
 * mod:<m>:<r> (x % m == r, integers) nonzero. The handle of a partition spec is also
 * the partition-scatter handle. Returns NULL on a malformed spec. */
parallax_kernel_t parallax_builtin_kernel(const char* spec);
/* 1 when `key` (a stdpar funnel key, e.g. "T parallax::detail::device_reduce(...) [with
 * T = float; ...]" or one of its ":scan" / ":add" / ... suffixed forms) names a kernel this
 * runtime provides built in, so a compiler need not register an image for it; 0 when the
 * key needs a registered image. Answered from the key alone, with or without a device
 * (parallax_kernel_lookup itself returns NULL when no device is available). */
int parallax_kernel_resolves(const char* key);

/* ---- arena residency ------------------------------------------------------------- */
enum parallax_residency {
    /* Default. The pinned host mirror is authoritative between calls: every ABI call
     * uploads the arena ranges it reads and downloads the ranges it writes, so host code
     * sees the reference's synchronous unified-memory behaviour. Small operands (at most
     * 64 KiB written, 256 KiB only read) are not copied at all: the kernel reads and writes
     * the host mirror itself (zero-copy). The device copy of a coherent block is therefore
     * not kept current. */
    PARALLAX_COHERENT = 0,
    /* The device copy is authoritative; ABI calls move nothing. Host code moves data
     * explicitly with parallax_arena_sync_to_device / _to_host (also when a block that
     * was used coherently becomes device-resident). */
    PARALLAX_DEVICE_RESIDENT = 1,
};
/* Applies to the whole arena block that contains ptr. Returns a parallax_status. */
int parallax_arena_set_residency(void* ptr, int mode);
int parallax_arena_get_residency(const void* ptr);
int parallax_arena_sync_to_device(const void* ptr, size_t bytes);
int parallax_arena_sync_to_host(void* ptr, size_t bytes);
/* dev_base + (ptr - host_base), or NULL when ptr is not in the arena. */
void* parallax_arena_device_ptr(const void* host_ptr);
void parallax_arena_bases(uint64_t* host_base, uint64_t* dev_base);
size_t parallax_arena_capacity(void);
size_t parallax_arena_used(void);      /* bytes currently allocated */
size_t parallax_arena_mapped(void);    /* bytes of device memory backing the arena */

/* ---- streams and asynchronous calls ---------------------------------------------- */
/* Thread-local CUDA stream for subsequent calls (NULL = the runtime's own per-thread
 * stream). */
int parallax_set_stream(void* cuda_stream);
/* Thread-local. With async != 0, ABI calls only enqueue work on the thread's stream and
 * return; outputs are valid after parallax_synchronize(). Host-memory operands are not
 * allowed in async mode (device pointers and DEVICE_RESIDENT arena blocks are). A
 * reduce `result` must then be a device pointer; copy_if returns SIZE_MAX and the
 * count is available from parallax_last_count() after synchronizing. */
int parallax_set_async(int async);
int parallax_synchronize(void);
size_t parallax_last_count(void);

/* ---- segmented primitives (batching) --------------------------------------------- */
/* No counterpart in the reference. `offsets` holds num_segments + 1 element offsets
 * (offsets[0] = 0, offsets[num_segments] = count) cutting `data` into segments; all
 * operands are DEVICE pointers (or PARALLAX_DEVICE_RESIDENT arena blocks). Each call is
 * one persistent launch over a tile work list (plus a one-CTA planner; partition adds a
 * count pass), tile shape (threads x vectors per thread) chosen by an autotuner on first
 * use, captured as a CUDA graph per argument set and replayed afterwards. Each returns a
 * parallax_status; synchronous unless async mode is on. Per segment, the result is the
 * plain primitive's result for that segment alone.
 *   reduce: results[s] = sum, max or min of segment s (0 for an empty segment);
 *     reduce:<sum|max|min> handle.
 *   exclusive_scan: per segment, output[i] = init + sum of the segment's earlier
 *     elements; inclusive_scan: output[i] = sum of the segment's elements up to i; scan
 *     handle.
 *   copy_if: the kept elements of segment s are written, in order, to
 *     output[offsets[s] ...]; counts[s] = how many; copy_if / remove_if handle (any
 *     predicate, x % m == r included).
 *   partition: segment s of output holds the elements of segment s that satisfy the
 *     predicate, in order, then the others, in order (stable); counts[s] = how many
 *     satisfy it; partition handle.
 *   unique: the first element of every run of equal elements of segment s is written, in
 *     order, to output[offsets[s] ...]; counts[s] = how many; unique handle.
 *   sort: each segment sorted ascending in place (sort:<dtype> handle), or 8-byte
 *     (key << 32 | value) records sorted stably by key (sort_kv:u32 handle). */
int parallax_segmented_reduce(parallax_kernel_t kernel, const void* data, size_t count,
                              const uint64_t* offsets, size_t num_segments, void* results);
int parallax_segmented_exclusive_scan(parallax_kernel_t kernel, const void* input,
                                      void* output, size_t count, const uint64_t* offsets,
                                      size_t num_segments, const void* init);
int parallax_segmented_inclusive_scan(parallax_kernel_t kernel, const void* input,
                                      void* output, size_t count, const uint64_t* offsets,
                                      size_t num_segments);
int parallax_segmented_copy_if(parallax_kernel_t kernel, const void* input, void* output,
                               size_t count, const uint64_t* offsets, size_t num_segments,
                               uint64_t* counts);
int parallax_segmented_partition(parallax_kernel_t kernel, const void* input, void* output,
                                 size_t count, const uint64_t* offsets, size_t num_segments,
                                 uint64_t* counts);
int parallax_segmented_unique(parallax_kernel_t kernel, const void* input, void* output,
                              size_t count, const uint64_t* offsets, size_t num_segments,
                              uint64_t* counts);
int parallax_segmented_sort(parallax_kernel_t kernel, void* data, size_t count,
                            const uint64_t* offsets, size_t num_segments);

/* ---- allocation-free scan -------------------------------------------------------- */
/* No counterpart in the reference. For callers that cannot allocate device memory: code
 * running inside an allocation hook (a malloc / operator new interposer that routes the
 * heap into the arena would re-enter itself if the runtime allocated) or a process whose
 * device memory belongs to its own pool. Same result as parallax_scan (init == NULL,
 * inclusive) or parallax_exclusive_scan (init != NULL, exclusive with that init), from
 * `input` to `output` (may be the same buffer), both DEVICE pointers, on `cuda_stream`
 * (NULL = the legacy default stream); returns when the result is ready, with a
 * parallax_status.
 * The runtime allocates nothing for it: the look-back status lives in one static device
 * array of 384.25 KiB that every GPU loading this library holds until the process exits.
 * That caps count at 24576 tiles: 704,643,072 elements of a 4-byte type, 352,321,536 of
 * an 8-byte type; larger counts return PARALLAX_ERR_INVALID_ARGUMENT and touch nothing.
 * The first call on a device looks up that array's device address (once per device, with
 * the device current). All calls share
 * the array: calls that overlap on the GPU (other streams, other threads) race and must
 * be serialized by the caller. */
int parallax_scan_noalloc(parallax_kernel_t scan_kernel, const void* input, void* output,
                          size_t count, size_t elem_size, const void* init,
                          void* cuda_stream);

/* ---- serving loop (continuous batching) --------------------------------------------
 * No counterpart in the reference (its calls are synchronous, one at a time, and not
 * thread-safe: src/kernel/kernel_launcher.hpp:172-176). Scheduler threads take requests
 * from any number of host threads, admit them in arrival order while the in-flight byte
 * budget and the arena (for sort temporaries) allow, coalesce queued requests of the same
 * kind into one segmented launch over per-request descriptors, and overlap `lanes` such
 * batches on the device. Operands stay where they are: PARALLAX_DEVICE_RESIDENT arena
 * blocks or device memory. A request's result does not depend on what it was batched with
 * (integers bit-exact; floating point within the primitives' tolerance). */
typedef struct parallax_serve_config {
    uint32_t lanes;          /* batches in flight on the device (0: 8) */
    uint32_t max_batch;      /* requests per coalesced launch (0: 1024) */
    uint64_t solo_elements;  /* longer requests run alone (0: 2^18); sorts that take the
                                radix path (from 2^20 keys) always do */
    uint64_t inflight_bytes; /* admission budget: operand + temporary bytes of admitted,
                                unfinished requests (0: half the arena capacity) */
    uint32_t schedulers;     /* host threads that form and launch batches, each owning an
                                equal share of the lanes (0: 2, at most `lanes`) */
    uint32_t reserved;       /* 0 */
} parallax_serve_config;

#define PARALLAX_REQ_EXCLUSIVE 1u /* scan: exclusive with `init` (else inclusive) */

typedef struct parallax_request {
    parallax_kernel_t kernel; /* reduce:<op>:<dt>, scan:<dt>, sort:<dt>, sort_kv:u32,
                                 copy_if / remove_if / partition / unique handles */
    const void* input;        /* sort: the data, sorted in place */
    void* output;             /* scan (NULL: in place), compaction output */
    size_t count;
    const void* init;         /* exclusive scan init (element size bytes; NULL = 0) */
    void* result;             /* host memory written on completion: the reduce value
                                 (element size) or the kept count (uint64); may be NULL */
    uint32_t flags;           /* PARALLAX_REQ_* */
} parallax_request;

typedef struct parallax_serve_stats {
    uint64_t requests, batches, coalesced_requests, solo_batches, max_batch;
    uint64_t peak_inflight_bytes, memory_waits, inflight_bytes, queued;
    /* scheduler threads' time (ns, summed over threads): forming batches and launching them,
     * handing finished batches back to their requests */
    uint64_t launch_ns, complete_ns;
} parallax_serve_stats;

/* Starts the serving loop (cfg may be NULL: defaults); a no-op when it runs already. */
int parallax_serve_start(const parallax_serve_config* cfg);
/* Finishes every submitted request, then stops the loop. */
int parallax_serve_stop(void);
/* Queues a request; *ticket is waited on exactly once with parallax_serve_wait (or polled
 * with parallax_serve_poll until it reports the request finished). */
int parallax_serve_submit(const parallax_request* req, uint64_t* ticket);
/* Blocks until the request finished; returns its parallax_status and, when done_ns is not
 * NULL, its completion time on parallax_clock_ns()'s clock. */
int parallax_serve_wait(uint64_t ticket, uint64_t* done_ns);
/* Non-blocking wait: *finished = 0 and PARALLAX_OK while the request runs (the ticket stays
 * valid); once it has finished, *finished = 1 and the call returns what parallax_serve_wait
 * would (status, done_ns) and consumes the ticket. */
int parallax_serve_poll(uint64_t ticket, int* finished, uint64_t* done_ns);
/* submit + wait: the blocking call a client thread makes. */
int parallax_serve_call(const parallax_request* req);
int parallax_serve_get_stats(parallax_serve_stats* out);
/* CLOCK_MONOTONIC in nanoseconds (the clock of parallax_serve_wait's done_ns). */
uint64_t parallax_clock_ns(void);

/* ---- bounded in-kernel waits ------------------------------------------------------ */
/* Every in-kernel wait (look-back on a predecessor tile, a bulk copy's arrival) gives up
 * after a bounded number of polls, records a code the host reads, and lets the kernel
 * return: the call then fails with PARALLAX_ERR_DEVICE_SPIN and the CUDA context stays
 * usable. PARALLAX_WAIT_LIMIT=<polls> (read once per process) lowers the look-back limit
 * from its default of 4,194,304 polls. No counterpart in the reference, whose fence waits
 * have no limit (src/kernel/kernel_launcher.cpp:438-443).
 * parallax_check_bounded_wait runs one look-back whose predecessor never publishes, with
 * its wait limited to `polls` (1 .. 4,194,304) polls, and returns what the host read:
 * PARALLAX_ERR_DEVICE_SPIN when the wait gave up and the kernel returned as designed. */
int parallax_check_bounded_wait(uint32_t polls);

/* ---- instrumentation ------------------------------------------------------------- */
/* Number of runtime kernel launches issued by this process so far. */
uint64_t parallax_launch_count(void);
/* Per-kernel device timing: when enabled, every runtime launch is bracketed with CUDA
 * events on its stream (small overhead; off by default). parallax_profile_json waits for
 * the recorded launches, folds them into per-kernel totals, writes
 * {"kernel": {"launches", "ms", "alg_bytes"}} into buf and returns the full JSON length;
 * totals accumulate until parallax_profile_reset(). alg_bytes is the launch's minimum HBM
 * traffic (compaction kernels count their input only). */
void parallax_profile_enable(int on);
size_t parallax_profile_json(char* buf, size_t cap);
void parallax_profile_reset(void);
/* Device ordinal, SM count and device name; returns a parallax_status. */
int parallax_device_info(int* device, int* sm_count, char* name, size_t name_cap);

#ifdef __cplusplus
}
#endif

#endif /* PARALLAX_RUNTIME_EXT_H */
