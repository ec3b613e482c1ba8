// Internal host-side interfaces of the B200 parallax runtime: per-thread workspaces
// (stream, device scratch, pinned result slot), the device-resident arena, kernel
// handles, and the launchers of the sm_100a primitive kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>

#include <atomic>
#include <functional>
#include <map>
#include <mutex>
#include <string>
#include <vector>
#include <utility>

#include "common.cuh"
#include "parallax/runtime.h"
#include "parallax/runtime_ext.h"

#define PXB_EXPORT extern "C" __attribute__((visibility("default")))

namespace pxb {

// ---- errors ------------------------------------------------------------------------
void set_error(int status, const char* fmt, ...) __attribute__((format(printf, 2, 3)));
void set_ok();
int last_error();
bool cuda_ok(cudaError_t e, const char* what);  // records PARALLAX_ERR_CUDA on failure

// ---- device context ------------------------------------------------------------------
struct DeviceInfo {
    int device = -1;
    int sm_count = 0;
    int max_threads_per_sm = 0;
    size_t smem_per_sm = 0;
    char name[256] = {0};
};
// Initializes the CUDA device once (PARALLAX_DEVICE, default 0). False when no device.
bool ensure_device();
const DeviceInfo& device_info();
void count_launch(unsigned n = 1);
uint64_t launch_count();

// Optional per-launch device timing (parallax_profile_enable). When enabled, each
// launcher brackets its kernel with CUDA events on the launch stream and records the
// launch's algorithmic bytes (the minimum HBM traffic of the work it does), so achieved
// bandwidth per kernel comes from live events. Disabled: one predictable branch.
struct Workspace;
struct Handle;
class ProfScope {
  public:
    ProfScope(Workspace& ws, const char* kernel, uint64_t alg_bytes);
    ~ProfScope();

  private:
    Workspace* ws_ = nullptr;
    const char* name_ = nullptr;
    uint64_t bytes_ = 0;
    cudaEvent_t start_ = nullptr;
};

// Pinned, device-mapped slot the kernels write small results into (reduce scalars,
// kept counts, in-kernel wait-timeout codes) so a synchronous call needs no extra
// device-to-host copy.
struct HostSlot {
    uint64_t result[4];     // up to 32 bytes of reduce / search results
    uint64_t count[2];      // kept counts (copy_if / partition)
    int32_t spin_error;     // nonzero when a bounded in-kernel wait gave up
    int32_t pad[7];
};

// Offsets inside the small scratch region.
constexpr size_t kScratchSmall = 64 << 10;
struct ScratchOff {
    static constexpr size_t ticket = 0;        // reduce last-block ticket (self-resetting)
    static constexpr size_t num_true = 256;    // partition: count of the count pass
    static constexpr size_t counters = 512;    // persistent launches: tile claim / exit (self-resetting)
    static constexpr size_t partials = 1024;   // reduce per-block partials (<= 48 KiB)
};

// Per-host-thread execution state. Every ABI call from a thread runs on that thread's
// stream, so calls from different threads overlap on the device.
struct Workspace {
    cudaStream_t own_stream = nullptr;
    cudaStream_t user_stream = nullptr;   // parallax_set_stream override
    bool async = false;
    void* d_scratch = nullptr;            // grows on demand, zeroed on (re)allocation
    size_t scratch_cap = 0;
    uint32_t epoch = 1;                   // look-back flag epoch, see next_epoch()
    HostSlot* h_slot = nullptr;
    HostSlot* d_slot = nullptr;           // device alias of h_slot
    size_t last_count = 0;
    // staging for operands that are plain (pageable) host pointers
    void* d_stage[3] = {nullptr, nullptr, nullptr};
    size_t stage_cap[3] = {0, 0, 0};
    cudaEvent_t done = nullptr;

    void* d_temp = nullptr;               // bulk temporaries (sort ping-pong buffer)
    size_t temp_cap = 0;
    void* d_seg = nullptr;                // segmented launches: counters, work list, partials
    size_t seg_cap = 0;
    void* d_seg_status = nullptr;         // segmented launches: look-back status entries only
    size_t seg_status_cap = 0;            // in entries
    void* d_radix = nullptr;              // radix sort: tile claim counters, digit histograms,
    size_t radix_cap = 0;                 // per-(tile, digit) look-back words
    uint32_t radix_epoch = 1;             // next epoch of those words, see next_radix_epochs()
    void* d_seg_radix = nullptr;          // segmented radix sort: counters (device-side epoch)
    size_t seg_radix_cap = 0;             // and per-(work item, digit) look-back words
    // Copy streams of calls whose host operand copies overlap their kernels (uploads and
    // downloads on separate copy engines) and the events that order them; see copy_streams().
    cudaStream_t copy_up = nullptr;
    cudaStream_t copy_down = nullptr;
    cudaEvent_t ev_copy[4] = {nullptr, nullptr, nullptr, nullptr};
    // Bumped whenever a workspace buffer is reallocated: cached graphs captured with older
    // buffer addresses are re-captured.
    uint64_t generation = 0;
    std::map<std::string, std::pair<uint64_t, cudaGraphExec_t>> graphs;
    // A transform2 of a transform_reduce / count_if funnel whose image can be fused with
    // the reduce that follows it: held back until the next call on this thread, which
    // either is that reduce (one fused pass) or runs it first (see abi.cu).
    struct Deferred {
        Handle* h = nullptr;
        void* in = nullptr;
        void* out = nullptr;
        size_t n = 0, in_es = 0, out_es = 0;
    } deferred;

    cudaStream_t stream() const { return user_stream ? user_stream : own_stream; }
    // Device scratch with a fixed layout (zeroed whenever it is reallocated):
    //   [0, kScratchSmall)   reduce tickets / partials / partition count (ScratchOff)
    //   [kScratchSmall, ...) look-back status entries, `tiles` of them
    // The regions never overlap, so a status word can only ever hold a status word.
    char* scratch(uint64_t tiles);
    void* temp(size_t bytes);
    void* seg(size_t bytes);  // zeroed on (re)allocation
    // Status entries of segmented look-backs, which carry the device-side epoch kept in the
    // segment buffer. A buffer of their own (zeroed on (re)allocation) so no other data
    // ever lies where a status word is read.
    void* seg_status(uint64_t entries);
    // Radix sort buffer (zeroed on (re)allocation): only radix-sort words ever live there.
    void* radix(size_t bytes);
    // Segmented radix sort buffer (zeroed on (re)allocation): its look-back words carry a
    // device-side epoch (replayed graphs advance it), so they never share the radix buffer,
    // whose words carry host-side epochs.
    void* seg_radix(size_t bytes);
    // `count` consecutive 22-bit epochs (one per radix pass) for the radix sort's look-back
    // words; returns the first. Called before a sort enqueues anything: on wrap-around it
    // enqueues a clear of the buffer, so no stale word can alias a reused epoch.
    uint32_t next_radix_epochs(uint32_t count);
    void* stage(int slot, size_t bytes);
    // Creates the copy streams and events on first use; false when that fails.
    bool copy_streams();
    // Look-back status words carry the launch epoch, so stale words from earlier
    // launches read as "not ready" without clearing the array between launches.
    uint32_t next_epoch();
};
Workspace* workspace();  // the calling thread's; nullptr when the device is unavailable
Workspace* current_workspace();  // the calling thread's if it has one, else nullptr
Workspace* new_workspace();  // an independent one (own stream and buffers), never freed

// Replays the CUDA graph cached under `key` on the workspace stream, capturing it first
// (thread-local capture of what `enqueue` puts on the stream) when it is missing or was
// captured before a buffer reallocation. `enqueue` must not grow workspace buffers.
// Falls back to plain enqueueing when PARALLAX_GRAPHS=0 or the stream is being captured
// by the caller (a parallax_set_stream stream inside the caller's own capture).
bool graph_launch(Workspace& ws, const std::string& key, const std::function<bool()>& enqueue);

// Waits for all work on the thread's stream with a deadline (PARALLAX_SYNC_TIMEOUT_MS,
// default 120000) and surfaces in-kernel wait timeouts. Returns a parallax_status.
int sync_stream(Workspace& ws);

// ---- heap pool (heap_pool.cu) --------------------------------------------------------
void* heap_pool_base();          // nullptr until the pool is initialized
size_t heap_pool_reservation();
size_t heap_pool_high_water();

// ---- arena ---------------------------------------------------------------------------
struct ArenaBlock {
    size_t offset = 0;
    size_t size = 0;
    int residency = 0;  // parallax_residency
};
bool arena_contains(const void* p);
// Looks up the block containing p; false when p is not inside a live block.
bool arena_find(const void* p, ArenaBlock* out);
void* arena_dev(const void* host_p);  // relocation dev_base + (p - host_base)
uint64_t arena_host_base();
uint64_t arena_dev_base();
uint64_t arena_mapped_bytes();  // bytes of the arena currently backed by device memory
// Copies every PARALLAX_COHERENT block (merged into contiguous ranges) host -> device or
// device -> host on the workspace stream. Kernels that dereference stored arena pointers
// may touch any block, so they get the reference's whole-arena coherence
// (src/memory/arena.cpp:296-304) restricted to blocks in coherent mode.
bool arena_sync_coherent(Workspace& ws, bool to_device);
// Pool-backed (whole-heap capture) mode: arena memory is page-locked host memory that
// kernels use in place (device address == host address); nothing is ever copied.
bool arena_zero_copy();
// Page-locks the host mirror under [p, p + bytes) if needed; true when a kernel can then
// access it through the host address itself (registered memory, host pointers usable).
bool arena_host_mapped(const void* p, size_t bytes);
// In that mode, page-locks the pool up to its high-water mark before a kernel may touch
// it; true (and nothing to do) otherwise.
bool arena_make_accessible();
// Host mirror <-> device copy of an arena range (split at page-lock chunk boundaries).
bool arena_copy_async(void* dst, const void* src, size_t bytes, bool to_device,
                      cudaStream_t s);

// ---- operands --------------------------------------------------------------------------
// How an ABI pointer reaches the device:
//   ARENA_COHERENT  arena block; range uploaded before / downloaded after the call
//   ARENA_RESIDENT  arena block in PARALLAX_DEVICE_RESIDENT mode; used in place
//   DEVICE          a CUDA device (or managed) pointer; used in place
//   HOST            any other host pointer; staged through device memory, results are
//                   copied back (the reference never copies results back to such
//                   pointers: src/memory/unified_buffer.cpp:126-136)
// ARENA_MAPPED: a small coherent arena operand that the kernel reads and writes in the
// page-locked host mirror itself (zero-copy), instead of a staged device copy.
enum class OperandKind { ARENA_COHERENT, ARENA_RESIDENT, ARENA_MAPPED, DEVICE, HOST };
struct Operand {
    void* user = nullptr;
    void* dev = nullptr;
    size_t bytes = 0;
    OperandKind kind = OperandKind::DEVICE;
};
// Resolves `p` and, when `upload`, enqueues the host-to-device copy. `stage_slot`
// selects the workspace staging buffer used for HOST operands.
bool resolve_operand(Workspace& ws, void* p, size_t bytes, bool upload, int stage_slot,
                     Operand* out,
                     bool mappable = true, size_t mapped_max = 0);
// Enqueues the device-to-host copy of the first `bytes` of a written operand.
bool writeback_operand(Workspace& ws, const Operand& op, size_t bytes);

// ---- kernel handles ----------------------------------------------------------------------
enum class Kind : int {
    NONE = 0,
    REDUCE, SCAN, SCAN_ADD, EXSCAN_SHIFT, SORT, SORT_KV,
    COMPACT_FLAGS,     // copy_if / remove_if predicate flags
    UNIQUE_FLAGS,      // adjacent-difference flags
    COMPACT_SCATTER,   // copy_if scatter
    PARTITION_SCATTER, // partition scatter: writes every element
    COUNT_IF, FIND, ARGMINMAX, MISMATCH,
    MAP,               // built-in element-wise op
    USER,              // sm_100a image loaded from a registered / loaded cubin
};
enum class RedOp : int { SUM = 0, MAX = 1, MIN = 2 };
// FLAGS: the element is kept when its byte in a flags array (written by a registered
// `:flags` image, one byte per element, nonzero = keep) is nonzero.
enum class PredKind : int { NONE = 0, GT, GE, LT, LE, EQ, NE, MOD, NONZERO, ODD_NONZERO, FLAGS };
struct Pred {
    PredKind kind = PredKind::NONE;
    bool negate = false;   // remove_if keeps elements for which the predicate is false
    double f = 0.0;        // operand for float element types
    int64_t i = 0;         // operand for signed integer element types
    uint64_t u = 0;        // operand for unsigned integer element types
    int64_t mod_m = 1, mod_r = 0;
    const uint8_t* flags = nullptr;  // FLAGS: device array of one byte per element
};
enum class MapOp : int { NONE = 0, SAXPY_GATHER_F32, AFFINE_F32, DOUBLE_PLUS_ONE_F32 };

struct Handle {
    Kind kind = Kind::NONE;
    DType dtype = DType::INVALID;
    RedOp op = RedOp::SUM;
    Pred pred;
    MapOp map = MapOp::NONE;
    bool remove = false;      // remove_if flavour of COMPACT_FLAGS
    // USER kernels
    cudaLibrary_t library = nullptr;
    cudaKernel_t kernel = nullptr;
    std::string name;
    std::vector<unsigned char> image;   // the registered image (linked again for fusion)
    std::vector<char> linked;           // cubin nvJitLink made of it, when loaded that way
    // Fused transform + reduce (fused.cu): 0 not tried, 1 linked, 2 not possible
    int fused_state = 0;
    cudaLibrary_t fused_library = nullptr;
    cudaKernel_t fused[6] = {};         // per reduced type: f32 f64 i32 i64 u32 u64
};
Handle* as_handle(parallax_kernel_t k);
Handle* builtin_handle(const char* spec);

// ---- run-time linking of registered images (fused.cu) ---------------------------------------
// Links fatbin / cubin / LTO-IR inputs for sm_100a with nvJitLink (link-time optimisation on)
// into one cubin; false when the link fails (with an error set unless `quiet`).
bool link_images(const std::vector<std::pair<const void*, size_t>>& inputs,
                 std::vector<char>* cubin, const char* what, bool quiet = false);
// True when `h` (a registered transform image) exports parallax_elem as LTO-IR, i.e. it
// links with the fused transform + reduce tile; links it on first use.
bool xform_fusable(Handle* h);
// One pass: reduce of xf(in[i]) over n input elements of in_es bytes into one element of
// dtype u at d_out (the runtime's reduce accumulation). xform_fusable(xf) must hold.
bool launch_xform_reduce(Workspace& ws, Handle* xf, DType u, const void* d_in, size_t n,
                         size_t in_es, void* d_out);
// Runs a transform held back on the calling thread (Workspace::deferred), if any.
void settle_deferred_here();

// ---- launchers (all asynchronous on `s`) -------------------------------------------------
// Reduce: writes one element (type of dtype; sum of f32 is rounded from fp64) to d_out.
bool launch_reduce(Workspace& ws, DType t, RedOp op, const void* d_in, size_t n, void* d_out);
// Inclusive (init == nullptr) or exclusive scan; in-place allowed.
// Scan of host arena operands (page-locked mirror addresses h_in / h_out, either may be null
// for a device-resident side) whose host-device copies overlap the scan: the tiles run in
// chunks, each chunk's upload and download on the workspace's copy streams.
bool launch_scan_copies(Workspace& ws, DType t, bool exclusive, const void* h_in,
                        const void* d_in, void* h_out, void* d_out, size_t n,
                        const void* init_host);
bool launch_scan(Workspace& ws, DType t, bool exclusive, const void* d_in, void* d_out,
                 size_t n, const void* init_host);
enum class CompactMode : int { SELECT = 0, UNIQUE = 1, PARTITION = 2 };
// Writes the kept count (uint64) to d_count.
bool launch_compact(Workspace& ws, DType t, CompactMode mode, const Pred& p, const void* d_in,
                    void* d_out, size_t n, uint64_t* d_count);
bool launch_count_if(Workspace& ws, DType t, const Pred& p, const void* d_in, size_t n,
                     uint64_t* d_count);
// Number of nonzero bytes of a flags array (partition with a registered `:flags` image).
bool launch_count_flags(Workspace& ws, const uint8_t* d_flags, size_t n, uint64_t* d_count);
// Elements a flags array written for launch_compact with PredKind::FLAGS must be padded to
// (the compaction reads whole rows of flags; bytes past n are ignored).
size_t compact_flags_padding(size_t n);
// by_key: 8-byte (key << 32 | value) records sorted stably by key (sort_kv handles).
bool launch_sort(Workspace& ws, DType t, void* d_data, size_t n, bool by_key = false);
// Smallest array launch_sort gives to the radix sort (by default; PARALLAX_SORT overrides).
size_t sort_radix_min(DType t);
// One-sweep LSD radix sort (kernels/radix.cu); launch_sort picks it for large arrays.
bool launch_radix_sort(Workspace& ws, DType t, void* d_data, size_t n, bool by_key = false);
bool launch_map(Workspace& ws, MapOp op, const void* d_in, void* d_out, size_t n,
                const void* captures, size_t capture_size);
bool launch_find(Workspace& ws, DType t, const Pred& p, const void* d_in, size_t n,
                 uint64_t* d_index);
bool launch_argminmax(Workspace& ws, DType t, bool want_max, bool want_last, const void* d_in,
                      size_t n, uint64_t* d_index);
bool launch_mismatch(Workspace& ws, DType t, const void* d_a, const void* d_b, size_t n,
                     uint64_t* d_index);

// Segmented launches over per-segment descriptors (SegDesc, segplan.cuh; a device-resident
// table of S entries whose lengths sum to `total`): one planner + one persistent kernel,
// asynchronous on the workspace stream, no graph capture. Used by the serving loop.
enum class SegKind : int { REDUCE = 0, SCAN = 1, COPY_IF = 2 };
struct SegDesc;
// `red` picks the reduce (sum / max / min); `mode` the compaction (select, unique,
// partition; partition counts into each descriptor's aux slot, then scatters).
bool launch_segmented_descs(Workspace& ws, SegKind op, DType t, const Pred& p, bool inclusive,
                            uint64_t init_bits, const SegDesc* d_descs, uint64_t S,
                            uint64_t total, RedOp red = RedOp::SUM,
                            CompactMode mode = CompactMode::SELECT);
// Sorts every descriptor's segment in place (aux = an n-element device temporary);
// `max_len` bounds the segment lengths. `t` is U64 for sort_kv records.
bool launch_segmented_sort_descs(Workspace& ws, DType t, const SegDesc* d_descs, uint64_t S,
                                 uint64_t total, uint64_t max_len, bool by_key = false);

// Device address of an operand of the segmented entry points, which take device memory or
// PARALLAX_DEVICE_RESIDENT arena blocks only. nullptr (error recorded) otherwise.
void* device_operand(const void* p, const char* fn, const char* what);

}  // namespace pxb
