// The parallax C ABI on top of the sm_100a launchers.
//
// Replaces the reference ABI forwarders (src/kernel/cache.cpp:106-392) and the
// KernelLauncher primitive schedules (src/kernel/kernel_launcher.cpp:277-1791). Each
// reference primitive is a chain of dispatches with a submit + fence wait per pass and
// host read-backs in between; here each primitive is one or two kernel launches on the
// calling thread's stream, followed by one bounded wait.
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <limits>

#include "parallax/kernel_abi.h"
#include "runtime.hpp"

namespace pxb {

// Coherent arena operands up to these sizes are used in place in the page-locked host
// mirror (zero-copy: the kernel's loads and stores cross PCIe) instead of being copied to the
// device and back, which for small operands costs more than the transfer itself. Measured per
// synchronous call: a 256 KiB fp32 reduce 23.8 us zero-copy against 28.7 us staged, a 256 KiB
// exclusive scan (read and written) 43.6 against 41.0 us, at 4 KiB 19.1 against 30.2 us.
constexpr size_t kMappedMax = size_t(64) << 10;       // operands a call writes
constexpr size_t kMappedMaxRead = size_t(256) << 10;  // operands a call only reads

bool resolve_operand(Workspace& ws, void* p, size_t bytes, bool upload, int slot,
                     Operand* out, bool mappable, size_t mapped_max) {
    out->user = p;
    out->bytes = bytes;
    if (!p) {
        set_error(PARALLAX_ERR_INVALID_ARGUMENT, "null buffer");
        return false;
    }
    cudaStream_t s = ws.stream();
    if (arena_contains(p)) {
        ArenaBlock b;
        if (!arena_find(p, &b)) {
            set_error(PARALLAX_ERR_INVALID_ARGUMENT, "pointer %p is inside the arena but not in "
                      "a live block", p);
            return false;
        }
        size_t off = static_cast<char*>(p) - reinterpret_cast<char*>(arena_host_base());
        if (off + bytes > b.offset + b.size) {
            set_error(PARALLAX_ERR_INVALID_ARGUMENT,
                      "operand of %zu bytes at %p overruns its arena block", bytes, p);
            return false;
        }
        out->dev = arena_dev(p);
        if (arena_zero_copy()) {  // whole-heap capture: used in place, nothing to copy
            out->kind = OperandKind::ARENA_RESIDENT;
            return arena_make_accessible();
        }
        out->kind = b.residency == PARALLAX_DEVICE_RESIDENT ? OperandKind::ARENA_RESIDENT
                                                            : OperandKind::ARENA_COHERENT;
        if (out->kind == OperandKind::ARENA_COHERENT && mappable && !ws.async &&
            bytes <= (mapped_max ? mapped_max : kMappedMax) && arena_host_mapped(p, bytes)) {
            // small: the kernel works on the host mirror itself, no copy either way
            out->kind = OperandKind::ARENA_MAPPED;
            out->dev = p;
            return true;
        }
        if (out->kind == OperandKind::ARENA_COHERENT && upload && bytes)
            return arena_copy_async(out->dev, p, bytes, true, s);
        return true;
    }
    cudaPointerAttributes attr;
    if (cudaPointerGetAttributes(&attr, p) == cudaSuccess &&
        (attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged)) {
        out->dev = attr.devicePointer ? attr.devicePointer : p;
        out->kind = OperandKind::DEVICE;
        return true;
    }
    cudaGetLastError();
    if (ws.async) {
        set_error(PARALLAX_ERR_INVALID_ARGUMENT,
                  "host pointer %p passed in async mode (use device or arena memory)", p);
        return false;
    }
    out->kind = OperandKind::HOST;
    out->dev = ws.stage(slot, bytes ? bytes : 16);
    if (!out->dev) return false;
    if (upload && bytes)
        return cuda_ok(cudaMemcpyAsync(out->dev, p, bytes, cudaMemcpyHostToDevice, s),
                       "operand staging upload");
    return true;
}

bool writeback_operand(Workspace& ws, const Operand& op, size_t bytes) {
    if (!bytes) return true;
    if (op.kind == OperandKind::ARENA_COHERENT)
        return arena_copy_async(op.user, op.dev, bytes, false, ws.stream());
    if (op.kind == OperandKind::HOST)
        return cuda_ok(cudaMemcpyAsync(op.user, op.dev, bytes, cudaMemcpyDeviceToHost,
                                       ws.stream()),
                       "operand download");
    return true;
}

}  // namespace pxb

using namespace pxb;

namespace {

void settle_deferred(Workspace& ws);

// Common prologue: handle + workspace + element-size check. A transform held back on this
// thread (Workspace::deferred) runs first.
Workspace* begin(Handle* h, const char* fn, size_t elem_size, std::initializer_list<Kind> kinds) {
    set_ok();
    if (Workspace* cur = current_workspace()) settle_deferred(*cur);
    if (!h) {
        set_error(PARALLAX_ERR_INVALID_HANDLE, "%s: invalid kernel handle", fn);
        return nullptr;
    }
    bool kind_ok = false;
    for (Kind k : kinds) kind_ok |= h->kind == k;
    if (!kind_ok) {
        set_error(PARALLAX_ERR_INVALID_HANDLE, "%s: handle '%s' is not valid for this call", fn,
                  h->name.c_str());
        return nullptr;
    }
    if (elem_size && h->dtype != DType::INVALID && h->kind != Kind::MAP &&
        h->kind != Kind::USER && h->kind != Kind::SORT_KV && dtype_size(h->dtype) != elem_size) {
        set_error(PARALLAX_ERR_INVALID_ARGUMENT, "%s: elem_size %zu does not match handle '%s'",
                  fn, elem_size, h->name.c_str());
        return nullptr;
    }
    return workspace();
}

int finish(Workspace& ws) { return ws.async ? PARALLAX_OK : sync_stream(ws); }

// Operands from this size up whose host copies a synchronous scan overlaps with its tiles.
constexpr size_t kCopyOverlapMin = size_t(64) << 20;

// A pointer into a live arena block in coherent mode (the call copies it both ways).
bool coherent_arena(const void* p) {
    ArenaBlock b;
    return p && arena_contains(p) && !arena_zero_copy() && arena_find(p, &b) &&
           b.residency != PARALLAX_DEVICE_RESIDENT;
}
// Device memory a call uses in place: a device-resident arena block or a CUDA pointer.
bool in_place_device(const void* p) {
    if (!p) return false;
    if (arena_contains(p)) {
        ArenaBlock b;
        return arena_find(p, &b) && (arena_zero_copy() || b.residency == PARALLAX_DEVICE_RESIDENT);
    }
    cudaPointerAttributes attr;
    const bool dev = cudaPointerGetAttributes(&attr, p) == cudaSuccess &&
                     (attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged);
    cudaGetLastError();
    return dev;
}

// Grid for USER kernels (grid-stride contract in kernel_abi.h).
dim3 user_grid(size_t count) {
    size_t blocks = (count + 255) / 256;
    size_t cap = (size_t)device_info().sm_count * 16;
    if (blocks > cap) blocks = cap;
    if (blocks == 0) blocks = 1;
    return dim3((unsigned)blocks);
}

bool launch_user(Workspace& ws, Handle* h, void* d_in, void* d_out, size_t count,
                 size_t in_es, size_t out_es, const void* captures, size_t capture_size) {
    if (capture_size > PARALLAX_MAX_CAPTURE_BYTES) {
        set_error(PARALLAX_ERR_INVALID_ARGUMENT, "captures of %zu bytes exceed %d", capture_size,
                  PARALLAX_MAX_CAPTURE_BYTES);
        return false;
    }
    parallax_launch_args a;
    memset(&a, 0, sizeof a);
    a.in = d_in;
    a.out = d_out;
    a.count = count;
    a.in_elem_size = in_es;
    a.out_elem_size = out_es;
    a.host_base = arena_host_base();
    a.dev_base = arena_dev_base();
    a.capture_size = capture_size;
    if (capture_size && captures) memcpy(a.captures, captures, capture_size);
    void* args[] = {&a};
    count_launch();
    return cuda_ok(cudaLaunchKernel((const void*)h->kernel, user_grid(count), dim3(256), args, 0,
                                    ws.stream()),
                   "cudaLaunchKernel(parallax_entry)");
}

// Kernels that dereference stored arena pointers may read any arena block, not only their
// operands: before they run, every coherent block is uploaded. Kernels that may also
// write through such pointers (registered images, relocate_f32) download every coherent
// block afterwards. This is the reference's whole-arena flush / invalidate around a launch
// (src/kernel/kernel_launcher.cpp:39-51, src/memory/arena.cpp:296-304), limited to blocks
// in coherent mode; device-resident blocks never move.
bool reads_through_pointers(const Handle* h) {
    return h->kind == Kind::USER || h->map == MapOp::SAXPY_GATHER_F32 ||
           h->map == MapOp::DOUBLE_PLUS_ONE_F32;
}
bool writes_through_pointers(const Handle* h) {
    return h->kind == Kind::USER || h->map == MapOp::DOUBLE_PLUS_ONE_F32;
}

// In-place element-wise launch (launch / launch_with_captures).
void map_inplace(const char* fn, parallax_kernel_t kernel, void* buffer, size_t count,
                 size_t elem_size, void* captures, size_t capture_size) {
    Handle* h = as_handle(kernel);
    Workspace* ws = begin(h, fn, 0, {Kind::MAP, Kind::USER});
    if (!ws || count == 0) return;
    const bool chase = reads_through_pointers(h);
    if (chase && !arena_sync_coherent(*ws, true)) return;
    Operand op;
    size_t bytes = count * elem_size;
    // (a kernel that chases stored pointers syncs the whole arena: operands stay staged)
    if (!resolve_operand(*ws, buffer, bytes, !(chase && arena_contains(buffer)), 0, &op, !chase))
        return;
    bool ok = h->kind == Kind::USER
        ? launch_user(*ws, h, op.dev, op.dev, count, elem_size, elem_size, captures, capture_size)
        : launch_map(*ws, h->map, op.dev, op.dev, count, captures, capture_size);
    if (!ok) return;
    if (writes_through_pointers(h)) {
        if (!arena_sync_coherent(*ws, false)) return;
        if (op.kind == OperandKind::HOST && !writeback_operand(*ws, op, bytes)) return;
    } else if (!writeback_operand(*ws, op, bytes)) {
        return;
    }
    finish(*ws);
}

// Keys of the funnels whose transform feeds a '+' reduce of its output and nothing else
// (stdpar.hpp:245-293): device_transform_reduce<T, U, F> ":xform" and device_count_if<T,
// Pred> ":pred". The funnel frees the staging buffer right after the reduce and never reads
// it, so the two calls may run as one fused pass.
bool fusable_funnel_key(const std::string& k) {
    auto ends_with = [&](const char* suf) {
        const size_t n = strlen(suf);
        return k.size() >= n && k.compare(k.size() - n, n, suf) == 0;
    };
    return (k.find("device_transform_reduce") != std::string::npos && ends_with(":xform")) ||
           (k.find("device_count_if") != std::string::npos && ends_with(":pred"));
}

void map_transform(const char* fn, parallax_kernel_t kernel, void* in, void* out, size_t count,
                   size_t in_es, size_t out_es, void* captures, size_t capture_size,
                   bool may_defer = true) {
    Handle* h = as_handle(kernel);
    Workspace* ws = begin(h, fn, 0, {Kind::MAP, Kind::USER});
    if (!ws || count == 0) return;
    if (out_es == 0) out_es = in_es;
    if (may_defer && h->kind == Kind::USER && !ws->async && capture_size == 0 &&
        fusable_funnel_key(h->name) && xform_fusable(h)) {
        // held back: the funnel's reduce of `out` runs both as one pass (parallax_reduce);
        // any other call on this thread runs the transform first
        ws->deferred = {h, in, out, count, in_es, out_es};
        return;
    }
    const bool chase = reads_through_pointers(h);
    if (chase && !arena_sync_coherent(*ws, true)) return;
    Operand oi, oo;
    if (!resolve_operand(*ws, in, count * in_es, !(chase && arena_contains(in)), 0, &oi, !chase))
        return;
    if (!resolve_operand(*ws, out, count * out_es, false, 1, &oo, !chase)) return;
    bool ok = h->kind == Kind::USER
        ? launch_user(*ws, h, oi.dev, oo.dev, count, in_es, out_es, captures, capture_size)
        : launch_map(*ws, h->map, oi.dev, oo.dev, count, captures, capture_size);
    if (!ok) return;
    if (writes_through_pointers(h)) {
        if (!arena_sync_coherent(*ws, false)) return;
        if (oo.kind == OperandKind::HOST && !writeback_operand(*ws, oo, count * out_es)) return;
    } else if (!writeback_operand(*ws, oo, count * out_es)) {
        return;
    }
    finish(*ws);
}

void settle_deferred(Workspace& ws) {
    if (!ws.deferred.h) return;
    const Workspace::Deferred d = ws.deferred;
    ws.deferred = Workspace::Deferred();
    map_transform("parallax_kernel_launch_transform2", reinterpret_cast<parallax_kernel_t>(d.h),
                  d.in, d.out, d.n, d.in_es, d.out_es, nullptr, 0, false);
}

// The funnel's reduce of a held-back transform's output: one pass over the transform's
// input, with the operand handling of the transform it replaces (a registered image may
// read through stored arena pointers: every coherent block is uploaded before and
// downloaded after, as for the transform alone).
void fused_transform_reduce(Workspace& ws, const Workspace::Deferred& d, Handle* red,
                            void* result) {
    Handle* xf = d.h;
    if (!arena_sync_coherent(ws, true)) return;
    Operand oi;
    if (!resolve_operand(ws, d.in, d.n * d.in_es, !arena_contains(d.in), 0, &oi, false)) return;
    if (!launch_xform_reduce(ws, xf, red->dtype, oi.dev, d.n, d.in_es, ws.d_slot->result))
        return;
    if (!arena_sync_coherent(ws, false)) return;
    if (sync_stream(ws) != PARALLAX_OK) return;
    memcpy(result, ws.h_slot->result, dtype_size(red->dtype));
}

}  // namespace

namespace pxb {
void settle_deferred_here() {
    if (Workspace* cur = current_workspace()) settle_deferred(*cur);
}
}  // namespace pxb

// ---- element-wise launches ------------------------------------------------------------------

PXB_EXPORT void parallax_kernel_launch(parallax_kernel_t kernel, ...) {
    va_list ap;
    va_start(ap, kernel);
    void* buffer = va_arg(ap, void*);
    size_t count = va_arg(ap, size_t);
    size_t elem_size = va_arg(ap, size_t);
    va_end(ap);
    map_inplace("parallax_kernel_launch", kernel, buffer, count, elem_size, nullptr, 0);
}

PXB_EXPORT void parallax_kernel_launch_transform(parallax_kernel_t kernel, ...) {
    va_list ap;
    va_start(ap, kernel);
    void* in = va_arg(ap, void*);
    void* out = va_arg(ap, void*);
    size_t count = va_arg(ap, size_t);
    size_t elem_size = va_arg(ap, size_t);
    va_end(ap);
    map_transform("parallax_kernel_launch_transform", kernel, in, out, count, elem_size,
                  elem_size, nullptr, 0);
}

PXB_EXPORT void parallax_kernel_launch_transform2(parallax_kernel_t kernel, void* in_buffer,
                                                  void* out_buffer, size_t count,
                                                  size_t in_elem_size, size_t out_elem_size) {
    map_transform("parallax_kernel_launch_transform2", kernel, in_buffer, out_buffer, count,
                  in_elem_size, out_elem_size, nullptr, 0);
}

PXB_EXPORT void parallax_kernel_launch_transform2_captures(
    parallax_kernel_t kernel, void* in_buffer, void* out_buffer, size_t count,
    size_t in_elem_size, size_t out_elem_size, void* captures, size_t capture_size) {
    map_transform("parallax_kernel_launch_transform2_captures", kernel, in_buffer, out_buffer,
                  count, in_elem_size, out_elem_size, captures, capture_size);
}

PXB_EXPORT void parallax_kernel_launch_with_captures(parallax_kernel_t kernel, void* buffer,
                                                     size_t count, void* captures,
                                                     size_t capture_size, size_t elem_size) {
    map_inplace("parallax_kernel_launch_with_captures", kernel, buffer, count, elem_size,
                captures, capture_size);
}

// ---- reduce -----------------------------------------------------------------------------------

PXB_EXPORT void parallax_reduce(parallax_kernel_t kernel, void* data, size_t count,
                                size_t elem_size, void* result) {
    Handle* h = as_handle(kernel);
    if (Workspace* cur = current_workspace(); cur && cur->deferred.h) {
        const Workspace::Deferred d = cur->deferred;
        if (h && h->kind == Kind::REDUCE && h->op == RedOp::SUM && result && data == d.out &&
            count == d.n && elem_size == d.out_es && dtype_size(h->dtype) == d.out_es &&
            !cur->async) {
            cur->deferred = Workspace::Deferred();
            set_ok();
            fused_transform_reduce(*cur, d, h, result);
            return;
        }
    }
    Workspace* ws = begin(h, "parallax_reduce", elem_size, {Kind::REDUCE});
    if (!ws) return;
    if (!result) {
        set_error(PARALLAX_ERR_INVALID_ARGUMENT, "parallax_reduce: null result");
        return;
    }
    const size_t es = dtype_size(h->dtype);
    if (count == 0) {  // reference: zero bytes for an empty range (kernel_launcher.cpp:918)
        if (ws->async) cudaMemsetAsync(result, 0, es, ws->stream());
        else memset(result, 0, es);
        return;
    }
    Operand op;
    if (!resolve_operand(*ws, data, count * es, true, 0, &op, true, kMappedMaxRead)) return;
    void* d_out = result;
    if (ws->async) {
        cudaPointerAttributes attr;
        if (cudaPointerGetAttributes(&attr, result) != cudaSuccess ||
            attr.type != cudaMemoryTypeDevice) {
            cudaGetLastError();
            if (!arena_contains(result)) {
                set_error(PARALLAX_ERR_INVALID_ARGUMENT,
                          "parallax_reduce: async mode needs a device result pointer");
                return;
            }
            d_out = arena_dev(result);
        }
    } else {
        d_out = ws->d_slot->result;
    }
    if (!launch_reduce(*ws, h->dtype, h->op, op.dev, count, d_out)) return;
    if (ws->async) return;
    if (sync_stream(*ws) != PARALLAX_OK) return;
    memcpy(result, ws->h_slot->result, es);
}

// ---- scans ------------------------------------------------------------------------------------

PXB_EXPORT void parallax_scan(parallax_kernel_t scan_kernel, parallax_kernel_t add_kernel,
                              void* data, size_t count, size_t elem_size) {
    Handle* h = as_handle(scan_kernel);
    Workspace* ws = begin(h, "parallax_scan", elem_size, {Kind::SCAN});
    if (!ws) return;
    if (!as_handle(add_kernel)) {
        set_error(PARALLAX_ERR_INVALID_HANDLE, "parallax_scan: invalid add kernel");
        return;
    }
    if (count <= 1) return;  // identity (kernel_launcher.cpp:1291)
    size_t bytes = count * dtype_size(h->dtype);
    const bool overlap = !ws->async && bytes >= kCopyOverlapMin && coherent_arena(data);
    Operand op;
    if (!resolve_operand(*ws, data, bytes, !overlap, 0, &op)) return;
    if (overlap) {
        if (!launch_scan_copies(*ws, h->dtype, false, data, op.dev, data, op.dev, count, nullptr))
            return;
    } else {
        if (!launch_scan(*ws, h->dtype, false, op.dev, op.dev, count, nullptr)) return;
        if (!writeback_operand(*ws, op, bytes)) return;
    }
    finish(*ws);
}

PXB_EXPORT void parallax_exclusive_scan(parallax_kernel_t scan_kernel,
                                        parallax_kernel_t add_kernel,
                                        parallax_kernel_t shift_kernel, void* input,
                                        void* output, size_t count, size_t elem_size,
                                        const void* init) {
    Handle* h = as_handle(scan_kernel);
    Workspace* ws = begin(h, "parallax_exclusive_scan", elem_size, {Kind::SCAN});
    if (!ws) return;
    if (!as_handle(add_kernel) || !as_handle(shift_kernel)) {
        set_error(PARALLAX_ERR_INVALID_HANDLE, "parallax_exclusive_scan: invalid add/shift kernel");
        return;
    }
    if (count == 0) return;
    size_t bytes = count * dtype_size(h->dtype);
    uint64_t zero = 0;
    const bool in_c = coherent_arena(input), out_c = coherent_arena(output);
    const bool overlap = !ws->async && bytes >= kCopyOverlapMin && (in_c || out_c) &&
                         (in_c || in_place_device(input)) && (out_c || in_place_device(output));
    Operand oi, oo;
    if (!resolve_operand(*ws, input, bytes, !overlap, 0, &oi)) return;
    if (!resolve_operand(*ws, output, bytes, false, 1, &oo)) return;
    if (overlap) {
        if (!launch_scan_copies(*ws, h->dtype, true, in_c ? input : nullptr, oi.dev,
                                out_c ? output : nullptr, oo.dev, count, init ? init : &zero))
            return;
    } else {
        if (!launch_scan(*ws, h->dtype, true, oi.dev, oo.dev, count, init ? init : &zero)) return;
        if (!writeback_operand(*ws, oo, bytes)) return;
    }
    finish(*ws);
}

// ---- sort -------------------------------------------------------------------------------------

PXB_EXPORT void parallax_sort(parallax_kernel_t kernel, void* data, size_t count,
                              size_t elem_size) {
    Handle* h = as_handle(kernel);
    Workspace* ws = begin(h, "parallax_sort", elem_size, {Kind::SORT, Kind::SORT_KV});
    if (!ws) return;
    if (h->kind == Kind::SORT_KV && elem_size != 8) {
        set_error(PARALLAX_ERR_INVALID_ARGUMENT, "parallax_sort: sort_kv sorts 8-byte records");
        return;
    }
    if (count <= 1) return;
    size_t bytes = count * dtype_size(h->dtype);
    Operand op;
    if (!resolve_operand(*ws, data, bytes, true, 0, &op)) return;
    if (!launch_sort(*ws, h->dtype, op.dev, count, h->kind == Kind::SORT_KV)) return;
    if (!writeback_operand(*ws, op, bytes)) return;
    finish(*ws);
}

// ---- compaction -------------------------------------------------------------------------------

namespace {

// A handle registered under a key of the named stdpar funnel (e.g. "device_partition").
bool from_funnel(const Handle* h, const char* funnel) {
    return h && h->name.find(funnel) != std::string::npos;
}

}  // namespace

PXB_EXPORT size_t parallax_copy_if(parallax_kernel_t flags_kernel, parallax_kernel_t scan_kernel,
                                   parallax_kernel_t add_kernel, parallax_kernel_t scatter_kernel,
                                   void* input, void* output, size_t count, size_t elem_size,
                                   int elem_is_float) {
    (void)elem_is_float;  // the element type is carried by the handle (or elem_size)
    Handle* h = as_handle(flags_kernel);
    Workspace* ws = begin(h, "parallax_copy_if", elem_size,
                          {Kind::COMPACT_FLAGS, Kind::UNIQUE_FLAGS, Kind::PARTITION_SCATTER,
                           Kind::USER});
    if (!ws) return 0;
    Handle* sc = as_handle(scatter_kernel);
    if (!as_handle(scan_kernel) || !as_handle(add_kernel) || !sc) {
        set_error(PARALLAX_ERR_INVALID_HANDLE, "parallax_copy_if: invalid scan/add/scatter kernel");
        return 0;
    }
    if (count == 0) return 0;
    // A registered `:flags` image (a compiler-emitted predicate, reference
    // src/kernel/kernel_launcher.cpp:1734-1738) writes one byte per element, nonzero = keep
    // (for remove_if the compiler's flags kernel already flags the elements to keep); the
    // built-in single-pass compaction then consumes those bytes in place of its own
    // predicate. Partition is recognised by its scatter handle (built-in partition scatter,
    // or any handle registered under a device_partition key), as in the reference, where
    // the scatter kernel decides whether rejected elements are written
    // (kernel_launcher.cpp:1778-1785).
    const bool user = h->kind == Kind::USER;
    CompactMode mode = CompactMode::SELECT;
    Pred pred = h->pred;
    if (h->kind == Kind::UNIQUE_FLAGS) mode = CompactMode::UNIQUE;
    else if (h->kind == Kind::PARTITION_SCATTER || sc->kind == Kind::PARTITION_SCATTER ||
             (user && (from_funnel(h, "device_partition") || from_funnel(sc, "device_partition"))))
        mode = CompactMode::PARTITION;
    if (h->kind == Kind::COMPACT_FLAGS && h->remove) pred.negate = true;
    DType t = h->dtype;
    if (user) {
        // the elements are moved as raw 4- or 8-byte words
        if (elem_size != 4 && elem_size != 8) {
            set_error(PARALLAX_ERR_UNSUPPORTED,
                      "parallax_copy_if: a registered flags kernel needs 4- or 8-byte elements "
                      "(got %zu)", elem_size);
            return 0;
        }
        t = elem_size == 4 ? DType::U32 : DType::U64;
    }
    size_t es = dtype_size(t);
    size_t bytes = count * es;
    const bool chase = user;  // the image may read through stored arena pointers
    if (chase && !arena_sync_coherent(*ws, true)) return 0;
    Operand oi, oo;
    if (!resolve_operand(*ws, input, bytes, !(chase && arena_contains(input)), 0, &oi, !chase))
        return 0;
    if (!resolve_operand(*ws, output, bytes, false, 1, &oo, !chase)) return 0;
    if (user) {
        uint8_t* d_flags = static_cast<uint8_t*>(ws->temp(compact_flags_padding(count)));
        if (!d_flags) return 0;
        if (!launch_user(*ws, h, oi.dev, d_flags, count, es, 1, nullptr, 0)) return 0;
        pred = Pred();
        pred.kind = PredKind::FLAGS;
        pred.flags = d_flags;
    }
    uint64_t* d_count = reinterpret_cast<uint64_t*>(ws->d_slot->count);
    if (!launch_compact(*ws, t, mode, pred, oi.dev, oo.dev, count, d_count)) return 0;
    if (ws->async) return std::numeric_limits<size_t>::max();
    if (sync_stream(*ws) != PARALLAX_OK) return 0;
    size_t kept = ws->h_slot->count[0];
    ws->last_count = kept;
    size_t written = mode == CompactMode::PARTITION ? count : kept;
    if (oo.kind == OperandKind::ARENA_COHERENT || oo.kind == OperandKind::HOST) {
        if (!writeback_operand(*ws, oo, written * es)) return 0;
        if (sync_stream(*ws) != PARALLAX_OK) return 0;
    }
    return kept;
}

// ---- search family ------------------------------------------------------------------------------

PXB_EXPORT size_t parallax_argminmax(parallax_kernel_t kernel, void* data, size_t count,
                                     size_t elem_size, int is_float, int want_max,
                                     int want_last) {
    (void)is_float;
    Handle* h = as_handle(kernel);
    Workspace* ws = begin(h, "parallax_argminmax", elem_size, {Kind::ARGMINMAX, Kind::REDUCE});
    if (!ws) return count;
    if (count <= 1) return 0;  // reference kernel_launcher.cpp:994-995
    Operand op;
    if (!resolve_operand(*ws, data, count * dtype_size(h->dtype), true, 0, &op, true,
                         kMappedMaxRead))
        return count;
    uint64_t* d_idx = reinterpret_cast<uint64_t*>(ws->d_slot->result);
    if (!launch_argminmax(*ws, h->dtype, want_max != 0, want_last != 0, op.dev, count, d_idx))
        return count;
    if (ws->async) return std::numeric_limits<size_t>::max();
    if (sync_stream(*ws) != PARALLAX_OK) return count;
    return ws->h_slot->result[0];
}

PXB_EXPORT size_t parallax_find(parallax_kernel_t kernel, void* data, size_t count,
                                size_t elem_size, int negate, const void* value) {
    Handle* h = as_handle(kernel);
    Workspace* ws = begin(h, "parallax_find", elem_size, {Kind::FIND});
    if (!ws) return count;
    if (count == 0) return 0;
    Pred p = h->pred;
    if (negate) p.negate = !p.negate;
    if (value) {  // find(value): equality with the caller's element bytes
        switch (h->dtype) {
            case DType::F32: { float v; memcpy(&v, value, 4); p.f = v; break; }
            case DType::F64: { memcpy(&p.f, value, 8); break; }
            case DType::I32: { int32_t v; memcpy(&v, value, 4); p.i = v; break; }
            case DType::I64: { memcpy(&p.i, value, 8); break; }
            case DType::U32: { uint32_t v; memcpy(&v, value, 4); p.u = v; break; }
            case DType::U64: { memcpy(&p.u, value, 8); break; }
            default: break;
        }
        p.kind = PredKind::EQ;
    }
    Operand op;
    if (!resolve_operand(*ws, data, count * dtype_size(h->dtype), true, 0, &op, true,
                         kMappedMaxRead))
        return count;
    uint64_t* d_idx = reinterpret_cast<uint64_t*>(ws->d_slot->result);
    if (!launch_find(*ws, h->dtype, p, op.dev, count, d_idx)) return count;
    if (ws->async) return std::numeric_limits<size_t>::max();
    if (sync_stream(*ws) != PARALLAX_OK) return count;
    return ws->h_slot->result[0];
}

PXB_EXPORT size_t parallax_mismatch(parallax_kernel_t kernel, void* a, void* b, size_t count,
                                    size_t elem_size) {
    Handle* h = as_handle(kernel);
    Workspace* ws = begin(h, "parallax_mismatch", elem_size, {Kind::MISMATCH});
    if (!ws) return count;
    if (count == 0) return 0;
    size_t bytes = count * dtype_size(h->dtype);
    Operand oa, ob;
    if (!resolve_operand(*ws, a, bytes, true, 0, &oa, true, kMappedMaxRead)) return count;
    if (!resolve_operand(*ws, b, bytes, true, 1, &ob, true, kMappedMaxRead)) return count;
    uint64_t* d_idx = reinterpret_cast<uint64_t*>(ws->d_slot->result);
    if (!launch_mismatch(*ws, h->dtype, oa.dev, ob.dev, count, d_idx)) return count;
    if (ws->async) return std::numeric_limits<size_t>::max();
    if (sync_stream(*ws) != PARALLAX_OK) return count;
    return ws->h_slot->result[0];
}

// ---- external buffers -------------------------------------------------------------------------

// C++ linkage, as declared in the reference header (runtime.h:144-145). Page-locks the
// caller's range so staged copies of it run at full link speed.
__attribute__((visibility("default"))) bool parallax_register_buffer(void* ptr, size_t size) {
    if (!ptr || !size) return false;
    if (!ensure_device()) return false;
    if (arena_contains(ptr)) return true;
    cudaError_t e = cudaHostRegister(ptr, size, cudaHostRegisterDefault);
    if (e == cudaErrorHostMemoryAlreadyRegistered) {
        cudaGetLastError();
        return true;
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return true;
}
