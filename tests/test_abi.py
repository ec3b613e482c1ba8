"""The C-ABI library: it loads, exports every function the headers declare (the reference
ABI plus the additive entry points), and resolves kernel handles without a GPU. CPU only:
no call here launches device work."""
from __future__ import annotations

import ctypes as C
import subprocess

import pytest

# the reference ABI (include/parallax/runtime.h:15-113, :144-145 in parallax-runtime)
REFERENCE_ABI = [
    "parallax_umalloc", "parallax_ufree", "parallax_arena_alloc", "parallax_arena_free",
    "parallax_arena_contains", "parallax_heap_contains", "parallax_kernel_load",
    "parallax_kernel_launch", "parallax_kernel_launch_transform",
    "parallax_kernel_launch_transform2", "parallax_kernel_launch_transform2_captures",
    "parallax_reduce", "parallax_argminmax", "parallax_find", "parallax_mismatch",
    "parallax_scan", "parallax_exclusive_scan", "parallax_sort", "parallax_copy_if",
    "parallax_kernel_register", "parallax_kernel_lookup",
    "parallax_kernel_launch_with_captures",
]


def exported(px) -> set[str]:
    out = subprocess.run(["nm", "-D", "--defined-only", str(px.LIB_PATH)],
                         capture_output=True, text=True, check=True).stdout
    return {ln.split()[-1] for ln in out.splitlines() if ln.strip()}


def test_library_loads(lib):
    assert lib.parallax_launch_count() >= 0


def test_every_declared_function_is_exported(px):
    syms = exported(px)
    declared = px.declared_functions()
    assert set(REFERENCE_ABI) <= set(declared["runtime.h"])
    missing = [f for names in declared.values() for f in names
               if f not in syms and f != "parallax_register_buffer"]
    assert not missing, missing


def test_register_buffer_keeps_cxx_linkage(px):
    # Declared outside extern "C" in the reference header: a mangled C++ symbol.
    syms = exported(px)
    assert "_Z24parallax_register_bufferPvm" in syms
    assert "parallax_register_buffer" not in syms


def test_only_abi_symbols_are_exported(px):
    syms = {s for s in exported(px) if not s.startswith("_Z24parallax_register_buffer")}
    declared = {f for names in px.declared_functions().values() for f in names}
    extra = sorted(s for s in syms if s.startswith("parallax_") and s not in declared)
    assert not extra, extra


GCC_KEY = ("T parallax::detail::device_reduce(const T*, std::size_t, T) "
           "[with T = {t}; std::size_t = long unsigned int]")
CLANG_KEY = "T parallax::detail::device_reduce(const T *, std::size_t, T) [T = {t}]"


@pytest.mark.parametrize("t", ["float", "double", "int", "long", "unsigned int",
                               "long unsigned int", "long long int"])
def test_funnel_keys_resolve_to_builtins(lib, t):
    for k in (GCC_KEY, CLANG_KEY):
        assert lib.parallax_kernel_resolves(k.format(t=t).encode())
    scan = f"void parallax::detail::device_scan(const T*, T*, std::size_t) [with T = {t}; std::size_t = long unsigned int]"
    assert lib.parallax_kernel_resolves((scan + ":scan").encode())
    assert lib.parallax_kernel_resolves((scan + ":add").encode())
    ex = f"void parallax::detail::device_exclusive_scan(const T*, T*, std::size_t, T) [with T = {t}; std::size_t = long unsigned int]"
    for sfx in (":scan", ":add", ":shift"):
        assert lib.parallax_kernel_resolves((ex + sfx).encode())
    srt = f"void parallax::detail::device_sort(T*, std::size_t) [with T = {t}; std::size_t = long unsigned int]"
    assert lib.parallax_kernel_resolves(srt.encode())
    uq = f"std::size_t parallax::detail::device_unique(T*, std::size_t) [with T = {t}; std::size_t = long unsigned int]"
    for sfx in (":flags", ":scan", ":add", ":scatter"):
        assert lib.parallax_kernel_resolves((uq + sfx).encode())


def test_lookup_misses_without_a_device(lib):
    """With no device nothing can run: a lookup misses even for a built-in key, so the
    caller runs its host loop (as a reference lookup does when its kernel cannot load)."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    k = GCC_KEY.format(t="float").encode()
    assert lib.parallax_kernel_resolves(k)
    assert not lib.parallax_kernel_lookup(k)


def test_functor_funnels_miss_without_an_image(lib):
    key = ("std::size_t parallax::detail::device_copy_if(const T*, T*, std::size_t, Pred) "
           "[with T = int; Pred = main()::<lambda(int)>; std::size_t = long unsigned int]:flags")
    assert not lib.parallax_kernel_lookup(key.encode())
    assert not lib.parallax_kernel_resolves(key.encode())
    assert not lib.parallax_kernel_lookup(b"no such kernel")
    assert not lib.parallax_kernel_lookup(None)
    assert not lib.parallax_kernel_resolves(None)


@pytest.mark.parametrize("funnel,sig", [
    ("copy_if", "std::size_t parallax::detail::device_copy_if(const T*, T*, std::size_t, Pred)"),
    ("remove_if", "std::size_t parallax::detail::device_remove_if(T*, std::size_t, Pred)"),
    ("partition", "std::size_t parallax::detail::device_partition(T*, std::size_t, Pred)"),
])
def test_compaction_funnels_need_only_a_flags_image(lib, funnel, sig):
    """The scan / add / scatter kernels of a compaction funnel are generic and resolve to
    built-ins; only the predicate's `:flags` kernel needs a registered image, and without
    one it misses (so the funnel's `kf && ks && ka && kc` test sends it to the host)."""
    base = f"{sig} [with T = int; Pred = P{funnel}; std::size_t = long unsigned int]"
    for sfx in (":scan", ":add", ":scatter"):
        assert lib.parallax_kernel_resolves((base + sfx).encode()), sfx
    assert not lib.parallax_kernel_resolves((base + ":flags").encode())


def test_count_if_and_transform_reduce_reduce_keys_resolve(lib):
    cnt = ("long int parallax::detail::device_count_if(const T*, std::size_t, Pred) "
           "[with T = float; Pred = G; std::size_t = long unsigned int]")
    assert lib.parallax_kernel_resolves((cnt + ":reduce").encode())
    assert not lib.parallax_kernel_resolves((cnt + ":pred").encode())
    tr = ("U parallax::detail::device_transform_reduce(const T*, std::size_t, F) "
          "[with T = float; U = double; F = Sq; std::size_t = long unsigned int]")
    assert lib.parallax_kernel_resolves((tr + ":reduce").encode())
    assert not lib.parallax_kernel_resolves((tr + ":xform").encode())


def test_registered_spirv_for_a_functor_funnel_misses(lib):
    # A SPIR-V image cannot run here: a functor funnel key registered with one misses
    # (host fallback); a fixed primitive key still has its built-in kernel (the GPU test
    # test_gpu_abi.py::test_registered_spirv_for_fixed_funnel_still_resolves looks it up).
    words = (C.c_uint * 5)(0x07230203, 0x00010500, 0, 1, 0)
    key = GCC_KEY.format(t="double").encode()
    lib.parallax_kernel_register(key, words, 5)
    assert lib.parallax_kernel_resolves(key)
    fkey = b"void parallax::detail::device_invoke(T*, std::size_t, F) [with T = float; F = f]"
    lib.parallax_kernel_register(fkey, words, 5)
    assert not lib.parallax_kernel_lookup(fkey)


@pytest.mark.parametrize("spec,ok", [
    ("reduce:sum:f32", True), ("reduce:max:i64", True), ("reduce:min:u32", True),
    ("scan:f64", True), ("exclusive_scan:i32", True), ("sort:f32", True),
    ("sort_kv:u32", True), ("copy_if:i32:mod:3:0", True), ("copy_if:f32:gt:0.5", True),
    ("remove_if:i64:lt:0", True), ("partition:i32:lt:0", True), ("unique:i32", True),
    ("count_if:u64:nonzero", True), ("find:f64:eq:2.5", True), ("argminmax:f32", True),
    ("mismatch:i32", True), ("map:saxpy_gather_f32", True), ("map:affine_f32", True),
    ("reduce:avg:f32", False), ("scan:f16", False), ("copy_if:f32:mod:3:0", False),
    ("copy_if:i32:between:1", False), ("sort_kv:u64", False), ("map:nope", False), ("", False),
    ("copy_if:i32:mod:4294967296:0", False), ("count_if:u32:mod:0:0", False),
    ("copy_if:i64:mod:4294967296:0", True),
])
def test_builtin_specs(lib, spec, ok):
    h = lib.parallax_builtin_kernel(spec.encode())
    assert bool(h) == ok
    lib.parallax_clear_error()


def test_invalid_handle_is_reported_not_crashing(lib, px):
    lib.parallax_clear_error()
    buf = (C.c_float * 4)()
    out = (C.c_float * 1)()
    lib.parallax_reduce(None, buf, 4, 4, out)
    assert lib.parallax_last_error() == px.ERR_INVALID_HANDLE
    lib.parallax_clear_error()
    assert lib.parallax_copy_if(None, None, None, None, buf, buf, 4, 4, 1) == 0
    assert lib.parallax_argminmax(None, buf, 4, 4, 1, 0, 0) == 4
    lib.parallax_clear_error()


def test_kernel_abi_header_layout():
    # parallax_launch_args: 8 eight-byte fields + 256 capture bytes
    from pathlib import Path
    src = (Path(__file__).resolve().parents[1] / "include/parallax/kernel_abi.h").read_text()
    assert "PARALLAX_MAX_CAPTURE_BYTES 256" in src


def test_check_bounded_wait_rejects_a_poll_count_outside_its_range(lib, px):
    assert lib.parallax_check_bounded_wait(0) == px.ERR_INVALID_ARGUMENT
    assert lib.parallax_check_bounded_wait((1 << 22) + 1) == px.ERR_INVALID_ARGUMENT
    lib.parallax_clear_error()
