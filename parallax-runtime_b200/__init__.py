"""ctypes binding of libparallax-runtime.so, the B200 (sm_100a) parallax runtime.

This is the Python-side view of the same C ABI that compiler-emitted C++ links against
(include/parallax/runtime.h, additive entry points in include/parallax/runtime_ext.h).
The tests and bench.py call the primitives through it exactly as C++ callers do, so every
number and parity result goes through the product's C ABI. Nothing here computes on the
CPU: when the shared library has not been built this module raises instead of falling
back.

The directory name contains a hyphen, so import it by path:

    spec = importlib.util.spec_from_file_location("parallax_runtime_b200", ".../__init__.py")
"""
from __future__ import annotations

import ctypes as C
import os
import re
from pathlib import Path

PKG_DIR = Path(__file__).resolve().parent
ROOT = PKG_DIR.parent
LIB_PATH = PKG_DIR / "lib" / "libparallax-runtime.so"
INCLUDE_DIR = ROOT / "include"

# parallax_status
OK = 0
ERR_INVALID_HANDLE = 1
ERR_INVALID_ARGUMENT = 2
ERR_OUT_OF_MEMORY = 3
ERR_CUDA = 4
ERR_TIMEOUT = 5
ERR_DEVICE_SPIN = 6
ERR_UNSUPPORTED = 7
ERR_NO_DEVICE = 8

ERR_SHUTDOWN = 9

COHERENT = 0
DEVICE_RESIDENT = 1
REQ_EXCLUSIVE = 1

vp = C.c_void_p
sz = C.c_size_t
u64 = C.c_uint64


class ServeConfig(C.Structure):
    """parallax_serve_config"""
    _fields_ = [("lanes", C.c_uint32), ("max_batch", C.c_uint32),
                ("solo_elements", C.c_uint64), ("inflight_bytes", C.c_uint64),
                ("schedulers", C.c_uint32), ("reserved", C.c_uint32)]


class Request(C.Structure):
    """parallax_request"""
    _fields_ = [("kernel", vp), ("input", vp), ("output", vp), ("count", sz), ("init", vp),
                ("result", vp), ("flags", C.c_uint32)]


class ServeStats(C.Structure):
    """parallax_serve_stats"""
    _fields_ = [(n, C.c_uint64) for n in (
        "requests", "batches", "coalesced_requests", "solo_batches", "max_batch",
        "peak_inflight_bytes", "memory_waits", "inflight_bytes", "queued", "launch_ns",
        "complete_ns")]

# name -> (restype, argtypes); variadic launches are declared with their fixed part only.
_SIGNATURES = {
    "parallax_umalloc": (vp, [sz, C.c_uint]),
    "parallax_ufree": (None, [vp]),
    "parallax_arena_alloc": (vp, [sz, sz]),
    "parallax_arena_free": (None, [vp]),
    "parallax_arena_contains": (C.c_int, [vp]),
    "parallax_heap_contains": (C.c_int, [vp]),
    "parallax_kernel_load": (vp, [vp, sz]),
    "parallax_kernel_launch": (None, None),
    "parallax_kernel_launch_transform": (None, None),
    "parallax_kernel_launch_transform2": (None, [vp, vp, vp, sz, sz, sz]),
    "parallax_kernel_launch_transform2_captures": (None, [vp, vp, vp, sz, sz, sz, vp, sz]),
    "parallax_reduce": (None, [vp, vp, sz, sz, vp]),
    "parallax_argminmax": (sz, [vp, vp, sz, sz, C.c_int, C.c_int, C.c_int]),
    "parallax_find": (sz, [vp, vp, sz, sz, C.c_int, vp]),
    "parallax_mismatch": (sz, [vp, vp, vp, sz, sz]),
    "parallax_scan": (None, [vp, vp, vp, sz, sz]),
    "parallax_exclusive_scan": (None, [vp, vp, vp, vp, vp, sz, sz, vp]),
    "parallax_sort": (None, [vp, vp, sz, sz]),
    "parallax_copy_if": (sz, [vp, vp, vp, vp, vp, vp, sz, sz, C.c_int]),
    "parallax_kernel_register": (None, [C.c_char_p, vp, sz]),
    "parallax_kernel_lookup": (vp, [C.c_char_p]),
    "parallax_kernel_launch_with_captures": (None, [vp, vp, sz, vp, sz, sz]),
    # runtime_ext.h
    "parallax_last_error": (C.c_int, []),
    "parallax_error_string": (C.c_char_p, [C.c_int]),
    "parallax_clear_error": (None, []),
    "parallax_builtin_kernel": (vp, [C.c_char_p]),
    "parallax_kernel_resolves": (C.c_int, [C.c_char_p]),
    "parallax_arena_set_residency": (C.c_int, [vp, C.c_int]),
    "parallax_arena_get_residency": (C.c_int, [vp]),
    "parallax_arena_sync_to_device": (C.c_int, [vp, sz]),
    "parallax_arena_sync_to_host": (C.c_int, [vp, sz]),
    "parallax_arena_device_ptr": (vp, [vp]),
    "parallax_arena_bases": (None, [C.POINTER(u64), C.POINTER(u64)]),
    "parallax_arena_capacity": (sz, []),
    "parallax_arena_used": (sz, []),
    "parallax_arena_mapped": (sz, []),
    "parallax_set_stream": (C.c_int, [vp]),
    "parallax_set_async": (C.c_int, [C.c_int]),
    "parallax_synchronize": (C.c_int, []),
    "parallax_last_count": (sz, []),
    "parallax_launch_count": (u64, []),
    "parallax_profile_enable": (None, [C.c_int]),
    "parallax_profile_json": (sz, [C.c_char_p, sz]),
    "parallax_profile_reset": (None, []),
    "parallax_scan_noalloc": (C.c_int, [vp, vp, vp, sz, sz, vp, vp]),
    "parallax_check_bounded_wait": (C.c_int, [C.c_uint32]),
    "parallax_segmented_reduce": (C.c_int, [vp, vp, sz, vp, sz, vp]),
    "parallax_segmented_exclusive_scan": (C.c_int, [vp, vp, vp, sz, vp, sz, vp]),
    "parallax_segmented_inclusive_scan": (C.c_int, [vp, vp, vp, sz, vp, sz]),
    "parallax_segmented_copy_if": (C.c_int, [vp, vp, vp, sz, vp, sz, vp]),
    "parallax_segmented_partition": (C.c_int, [vp, vp, vp, sz, vp, sz, vp]),
    "parallax_segmented_unique": (C.c_int, [vp, vp, vp, sz, vp, sz, vp]),
    "parallax_segmented_sort": (C.c_int, [vp, vp, sz, vp, sz]),
    "parallax_device_info": (C.c_int, [C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_char_p, sz]),
    "parallax_serve_start": (C.c_int, [C.POINTER(ServeConfig)]),
    "parallax_serve_stop": (C.c_int, []),
    "parallax_serve_submit": (C.c_int, [C.POINTER(Request), C.POINTER(u64)]),
    "parallax_serve_wait": (C.c_int, [u64, C.POINTER(u64)]),
    "parallax_serve_poll": (C.c_int, [u64, C.POINTER(C.c_int), C.POINTER(u64)]),
    "parallax_serve_call": (C.c_int, [C.POINTER(Request)]),
    "parallax_serve_get_stats": (C.c_int, [C.POINTER(ServeStats)]),
    "parallax_clock_ns": (u64, []),
}

_lib = None


class ParallaxError(RuntimeError):
    def __init__(self, status: int, what: str):
        super().__init__(f"{what}: status {status}")
        self.status = status


def load(path: str | os.PathLike | None = None) -> C.CDLL:
    """Loads the runtime library (once) and declares every exported signature."""
    global _lib
    if _lib is not None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise RuntimeError(
            f"{p} is not built; run `python parallax-runtime_b200/build.py` "
            "(the runtime has no CPU fallback)")
    lib = C.CDLL(str(p))
    for name, (res, args) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        if args is not None:
            fn.argtypes = args
    _lib = lib
    return lib


def check(what: str = "parallax call") -> None:
    """Raises ParallaxError when the calling thread's last ABI call failed."""
    st = load().parallax_last_error()
    if st != OK:
        load().parallax_clear_error()
        raise ParallaxError(st, what)


def builtin(spec: str) -> int:
    h = load().parallax_builtin_kernel(spec.encode())
    if not h:
        raise ValueError(f"bad built-in kernel spec {spec!r}")
    return h


def declared_functions() -> dict[str, list[str]]:
    """Function names declared in include/parallax/*.h, per header."""
    out: dict[str, list[str]] = {}
    for h in sorted(INCLUDE_DIR.rglob("*.h")):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        text = re.sub(r"//[^\n]*", "", text)
        names = re.findall(r"\b(parallax_[a-z0-9_]+)\s*\(", text)
        out[h.name] = sorted(set(names))
    return out


def profile_json() -> dict:
    """Per-kernel launches / device ms / algorithmic bytes recorded since the last call."""
    import json
    lib = load()
    need = lib.parallax_profile_json(None, 0)
    buf = C.create_string_buffer(need + 1)
    lib.parallax_profile_json(buf, need + 1)
    return json.loads(buf.value.decode() or "{}")


def device_info() -> tuple[int, int, str]:
    d, s = C.c_int(), C.c_int()
    name = C.create_string_buffer(256)
    st = load().parallax_device_info(C.byref(d), C.byref(s), name, 256)
    if st != OK:
        raise ParallaxError(st, "parallax_device_info")
    return d.value, s.value, name.value.decode()
