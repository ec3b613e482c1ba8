"""The reference's unit-test known answers and golden vectors through the C ABI on a B200,
and the operand paths of the ABI: coherent arena blocks (host pointer in, host-visible
result out, like the reference's unified memory), device-resident arena blocks, raw
device pointers and plain host pointers."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import cases
from cases import F32_TOL, F64_TOL, SIZES, golden, same_as_golden
from helpers import Arena

pytestmark = pytest.mark.gpu


@pytest.fixture
def arena(lib):
    a = Arena(lib)
    yield a
    a.free()


def P(a: np.ndarray) -> int:
    return a.ctypes.data


# ---- known answers of the reference unit tests, through arena (unified) memory --------------
def test_kat_reduce(lib, px, arena):
    x, want = cases.kat_reduce()
    data = arena.array(x)
    result = np.array([-1.0], np.float32)
    lib.parallax_reduce(px.builtin("reduce:sum:f32"), P(data), data.size, 4, P(result))
    px.check()
    assert result[0] == want


def test_kat_scan(lib, px, arena):
    x, want = cases.kat_scan()
    data = arena.array(x)
    h = px.builtin("scan:f32")
    lib.parallax_scan(h, h, P(data), data.size, 4)
    px.check()
    assert np.array_equal(data, want)


def test_kat_sort(lib, px, arena):
    x = cases.kat_sort()
    data = arena.array(x)
    lib.parallax_sort(px.builtin("sort:f32"), P(data), data.size, 4)
    px.check()
    assert np.all(np.diff(data) >= 0)
    assert data.astype(np.uint64).sum() == x.astype(np.uint64).sum()


def test_kat_copy_if(lib, px, arena):
    x, wk, want = cases.kat_copy_if()
    inp = arena.array(x)
    out = arena.array(np.full(x.size, -1.0, np.float32))
    h = px.builtin("copy_if:f32:gt:0.5")
    k = lib.parallax_copy_if(h, h, h, h, P(inp), P(out), x.size, 4, 1)
    px.check()
    assert k == wk and np.array_equal(out[:k], want)
    assert np.all(out[k:] == -1.0)  # only the kept prefix is written


def test_kat_relocation(lib, px, arena):
    x, want = cases.kat_relocate()
    data = arena.array(x)
    cap = np.array([P(data)], np.uint64)  # the HOST address, relocated in the kernel
    lib.parallax_kernel_launch_with_captures(px.builtin("map:relocate_f32"), P(data), data.size,
                                             P(cap), 8, 4)
    px.check()
    assert np.all(data == want)


def test_kat_arena(lib):
    # tests/unit/test_arena.cpp:41-65
    a = lib.parallax_arena_alloc(1000 * 4, 16)
    b = lib.parallax_arena_alloc(500 * 4, 16)
    assert a and b and a % 256 == 0 and b % 256 == 0 and b > a
    assert lib.parallax_arena_contains(a) and lib.parallax_arena_contains(b)
    lib.parallax_arena_free(a)
    c = lib.parallax_arena_alloc(1000 * 4, 16)
    assert c == a  # freed block reused
    on_stack = C.c_int(42)
    assert not lib.parallax_arena_contains(C.addressof(on_stack))
    assert not lib.parallax_arena_alloc(lib.parallax_arena_capacity() + 4096, 256)
    lib.parallax_clear_error()
    lib.parallax_arena_free(b)
    lib.parallax_arena_free(c)


def test_arena_coalesces_freed_neighbours(lib):
    ps = [lib.parallax_arena_alloc(1 << 20, 256) for _ in range(4)]
    for p in ps:
        lib.parallax_arena_free(p)
    # the four freed neighbours merge into one 4 MiB hole, so first fit lands at or
    # before it instead of extending the arena
    big = lib.parallax_arena_alloc(4 << 20, 256)
    assert big <= ps[0]
    lib.parallax_arena_free(big)


# ---- golden vectors of the reference's CPU path, through the ABI ------------------------------
@pytest.mark.parametrize("n", SIZES)
def test_golden_vectors(lib, px, ox, dev, n):
    x = cases.inputs(n)
    g = golden()
    res = (C.c_ubyte * 8)()
    for t in ("i32", "i64"):
        d = dev.put(x[t])
        lib.parallax_reduce(px.builtin(f"reduce:sum:{t}"), d.data_ptr(), n, x[t].itemsize, res)
        px.check()
        assert np.frombuffer(bytes(res), x[t].dtype, 1)[0] == g[f"reduce_{t}_{n}"][0]
        h = px.builtin(f"scan:{t}")
        lib.parallax_scan(h, h, d.data_ptr(), n, x[t].itemsize)
        px.check()
        assert same_as_golden(f"inclusive_scan_{t}_{n}", dev.get(d, x[t].dtype, n))
        d = dev.put(x[t])
        o = dev.empty(x[t].nbytes)
        init = np.array([7], x[t].dtype)
        lib.parallax_exclusive_scan(h, h, h, d.data_ptr(), o.data_ptr(), n, x[t].itemsize, P(init))
        px.check()
        assert same_as_golden(f"exclusive_scan_{t}_{n}", dev.get(o, x[t].dtype, n))
    for t in ("u32", "i32"):
        d = dev.put(x[t])
        lib.parallax_sort(px.builtin(f"sort:{t}"), d.data_ptr(), n, 4)
        px.check()
        assert same_as_golden(f"sort_{t}_{n}", dev.get(d, x[t].dtype, n))
    d, o = dev.put(x["i32"]), dev.empty(x["i32"].nbytes)
    h = px.builtin("copy_if:i32:mod:3:0")
    k = lib.parallax_copy_if(h, h, h, h, d.data_ptr(), o.data_ptr(), n, 4, 0)
    assert same_as_golden(f"copy_if_mod3_i32_{n}", dev.get(o, np.int32, k))
    h = px.builtin("remove_if:i32:mod:3:0")
    k = lib.parallax_copy_if(h, h, h, h, d.data_ptr(), o.data_ptr(), n, 4, 0)
    assert same_as_golden(f"remove_if_mod3_i32_{n}", dev.get(o, np.int32, k))
    u = dev.put(cases.unique_input(x["i32"]))
    h = px.builtin("unique:i32")
    k = lib.parallax_copy_if(h, h, h, h, u.data_ptr(), o.data_ptr(), n, 4, 0)
    assert same_as_golden(f"unique_i32_{n}", dev.get(o, np.int32, k))
    h = px.builtin("partition:i32:lt:0")
    k = lib.parallax_copy_if(h, h, h, h, d.data_ptr(), o.data_ptr(), n, 4, 0)
    px.check()
    assert k == int(g[f"partition_neg_i32_{n}_k"][0])
    if n <= 5000:
        got = dev.get(o, np.int32, n)
        want = g[f"partition_neg_i32_{n}"]
        assert np.array_equal(np.sort(got[:k]), np.sort(want[:k]))
        assert np.array_equal(np.sort(got[k:]), np.sort(want[k:]))
    d = dev.put(x["f32"])
    res4 = (C.c_ubyte * 4)()
    lib.parallax_reduce(px.builtin("reduce:sum:f32"), d.data_ptr(), n, 4, res4)
    want = float(g[f"reduce_f32_{n}"][0])
    assert abs(np.frombuffer(bytes(res4), np.float32, 1)[0] - want) <= F32_TOL * abs(want)
    d = dev.put(x["f64"])
    lib.parallax_reduce(px.builtin("reduce:sum:f64"), d.data_ptr(), n, 8, res)
    want = float(g[f"reduce_f64_{n}"][0])
    assert abs(np.frombuffer(bytes(res), np.float64, 1)[0] - want) <= F64_TOL * abs(want)


# ---- operand paths ------------------------------------------------------------------------------
def test_host_pointer_operands_get_results_back(lib, px, ox):
    # The reference never copies results back to non-arena pointers
    # (src/memory/unified_buffer.cpp:126-136); here they are staged both ways.
    x = ox.gen("i32_pm1000", 12, 100001)
    data = x.copy()
    h = px.builtin("scan:i32")
    lib.parallax_scan(h, h, P(data), data.size, 4)
    px.check()
    assert np.array_equal(data, ox.scan(x))
    out = np.zeros_like(x)
    h = px.builtin("copy_if:i32:gt:0")
    k = lib.parallax_copy_if(h, h, h, h, P(x), P(out), x.size, 4, 0)
    want, wk = ox.compact(x, ox.COPY_IF, ox.P_GT, 0)
    assert k == wk and np.array_equal(out[:k], want[:k])


def test_coherent_arena_sees_host_writes_between_calls(lib, px, arena):
    data = arena.array(np.ones(10000, np.int64))
    res = np.zeros(1, np.int64)
    h = px.builtin("reduce:sum:i64")
    lib.parallax_reduce(h, P(data), data.size, 8, P(res))
    assert res[0] == 10000
    data[:] = 3  # host write through the arena pointer, no explicit sync
    lib.parallax_reduce(h, P(data), data.size, 8, P(res))
    assert res[0] == 30000


def test_device_resident_block_moves_nothing_until_synced(lib, px, arena):
    data = arena.array(np.arange(4096, dtype=np.int32))
    assert lib.parallax_arena_set_residency(P(data), px.DEVICE_RESIDENT) == 0
    assert lib.parallax_arena_get_residency(P(data)) == px.DEVICE_RESIDENT
    assert lib.parallax_arena_sync_to_device(P(data), data.nbytes) == 0
    h = px.builtin("scan:i32")
    lib.parallax_scan(h, h, P(data), data.size, 4)
    px.check()
    assert np.array_equal(data, np.arange(4096))  # host mirror untouched
    assert lib.parallax_arena_sync_to_host(P(data), data.nbytes) == 0
    assert np.array_equal(data, np.cumsum(np.arange(4096)))
    lib.parallax_arena_set_residency(P(data), px.COHERENT)


def test_arena_device_pointer_relocation(lib, arena):
    data = arena.array(np.zeros(16, np.float32))
    hb, db = C.c_uint64(), C.c_uint64()
    lib.parallax_arena_bases(C.byref(hb), C.byref(db))
    dp = lib.parallax_arena_device_ptr(P(data))
    assert dp == db.value + (P(data) - hb.value)
    assert not lib.parallax_arena_device_ptr(P(np.zeros(4)))


def test_saxpy_gather_with_relocation(lib, px, ox, arena):
    # transform2 over {float x; u32 pad; float* p} records, y = 1.5*x + *p
    n = 1 << 16
    tgt = arena.array(ox.gen("f32_unit", 21, n))
    idx = (ox.gen_u64(22, n) % np.uint64(n)).astype(np.uint64)
    rec = np.zeros(n * 4, np.uint32)
    rec[0::4] = ox.gen("f32_unit", 23, n).view(np.uint32)
    ptrs = np.uint64(P(tgt)) + idx * np.uint64(4)
    rec.view(np.uint64)[1::2] = ptrs
    recs = arena.array(rec)
    y = arena.empty(n, np.float32)
    a = np.array([1.5], np.float32)
    lib.parallax_kernel_launch_transform2_captures(px.builtin("map:saxpy_gather_f32"), P(recs),
                                                   P(y), n, 16, 4, P(a), 4)
    px.check()
    want = ox.saxpy_gather(rec, 1.5, np.array(tgt), P(tgt))
    assert np.array_equal(y, want)


def test_async_mode_with_device_result(lib, px, ox, dev):
    import torch
    x = ox.gen("i64_full", 30, 1 << 20)
    d = dev.put(x)
    r = torch.zeros(1, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()  # the runtime works on its own stream
    assert lib.parallax_set_async(1) == 0
    try:
        lib.parallax_reduce(px.builtin("reduce:sum:i64"), d.data_ptr(), x.size, 8, r.data_ptr())
        px.check()
        assert lib.parallax_synchronize() == 0
    finally:
        lib.parallax_set_async(0)
    assert int(r.item()) == int(ox.reduce_sum(x))


def test_elem_size_mismatch_is_rejected(lib, px, dev):
    d = dev.put(np.zeros(16, np.float32))
    out = (C.c_ubyte * 8)()
    lib.parallax_reduce(px.builtin("reduce:sum:f64"), d.data_ptr(), 16, 4, out)
    assert lib.parallax_last_error() == px.ERR_INVALID_ARGUMENT
    lib.parallax_clear_error()


def test_launch_counter_counts_kernels(lib, px, dev):
    d = dev.put(np.ones(1 << 16, np.float32))
    out = (C.c_ubyte * 4)()
    before = lib.parallax_launch_count()
    lib.parallax_reduce(px.builtin("reduce:sum:f32"), d.data_ptr(), 1 << 16, 4, out)
    assert lib.parallax_launch_count() == before + 1


def test_coherent_operand_spanning_arena_chunks(lib, px, ox, arena):
    # 600 MiB block: its range crosses a 512 MiB page-lock chunk of the host mirror
    n = (600 << 20) // 4
    x = ox.gen("i32_pm1000", 31, n)
    data = arena.array(x)
    res = np.zeros(1, np.int32)
    lib.parallax_reduce(px.builtin("reduce:sum:i32"), P(data), n, 4, P(res))
    px.check()
    assert res[0] == ox.reduce_sum(x)
    h = px.builtin("scan:i32")
    lib.parallax_scan(h, h, P(data), n, 4)
    px.check()
    assert np.array_equal(data, ox.scan(x))


GCC_REDUCE_KEY = ("T parallax::detail::device_reduce(const T*, std::size_t, T) "
                  "[with T = {t}; std::size_t = long unsigned int]")


def test_funnel_lookups_return_one_handle(lib):
    k = GCC_REDUCE_KEY.format(t="float").encode()
    h = lib.parallax_kernel_lookup(k)
    assert h and h == lib.parallax_kernel_lookup(k)


def test_registered_spirv_for_fixed_funnel_still_resolves(lib):
    # A SPIR-V image cannot run here; a fixed primitive funnel key resolves to the
    # built-in sm_100a kernel, a functor funnel key misses (host fallback).
    words = (C.c_uint * 5)(0x07230203, 0x00010500, 0, 1, 0)
    key = GCC_REDUCE_KEY.format(t="double").encode() + b" "
    lib.parallax_kernel_register(key, words, 5)
    assert lib.parallax_kernel_lookup(key)
    fkey = b"void parallax::detail::device_invoke(T*, std::size_t, F) [with T = double; F = g]"
    lib.parallax_kernel_register(fkey, words, 5)
    assert not lib.parallax_kernel_lookup(fkey)
    lib.parallax_clear_error()

