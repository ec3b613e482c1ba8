"""The allocation-free scan entry point, parallax_scan_noalloc, through the C ABI.

It exists for callers that cannot allocate device memory (code running inside an
allocation hook, or a process whose device memory belongs to its own pool): its look-back
status lives in a static device array instead of runtime-allocated scratch. Here it must
give the same result as the regular entry points (parallax_scan / parallax_exclusive_scan)
on two calls in a row - the second call runs with the array still holding the first
call's contents - and must refuse counts beyond its static capacity.

This file is collected last so that a run stopping at the first failure has already run
every other test; it also passes alone in a fresh process.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from cases import F32_TOL, F64_TOL

pytestmark = pytest.mark.gpu

MAX_TILES = 24576
TILE = {4: 28672, 8: 14336}  # elements per look-back tile of the scan kernel (112 KiB)


def gen(ox, t, n, seed):
    return {"f32": lambda: ox.gen("f32_unit", seed, n), "f64": lambda: ox.gen("f64_unit", seed, n),
            "i32": lambda: ox.gen("i32_pm1000", seed, n), "i64": lambda: ox.gen("i64_full", seed, n),
            "u32": lambda: ox.gen("u32_full", seed, n), "u64": lambda: ox.gen_u64(seed, n)}[t]()


def same(t, got, want):
    if t == "f32":
        return np.max(np.abs(got.astype(np.float64) - want) / np.maximum(np.abs(want), 1e-30)) <= F32_TOL
    if t == "f64":
        return np.max(np.abs(got - want) / np.maximum(np.abs(want), 1e-300)) <= F64_TOL
    return np.array_equal(got, want)


@pytest.mark.parametrize("t", ["f32", "f64", "i32", "i64", "u32", "u64"])
@pytest.mark.parametrize("n", [1, 3073, 1 << 20, (1 << 22) + 17])
@pytest.mark.parametrize("exclusive", [False, True])
def test_noalloc_matches_existing_entry_point(lib, px, ox, dev, t, n, exclusive):
    import torch
    x = gen(ox, t, n, seed=41)
    s = x.itemsize
    h = px.builtin(f"scan:{t}")
    init = np.array([3], dtype=x.dtype)
    # existing entry points (runtime-allocated scratch)
    d_ref = dev.put(x)
    if exclusive:
        o_ref = dev.empty(x.nbytes)
        lib.parallax_exclusive_scan(h, h, h, d_ref.data_ptr(), o_ref.data_ptr(), n, s,
                                    init.ctypes.data)
    else:
        lib.parallax_scan(h, h, d_ref.data_ptr(), n, s)
        o_ref = d_ref
    px.check("existing entry point")
    want = dev.get(o_ref, x.dtype, n)
    # allocation-free entry point, twice in a row on the caller's stream
    d_in = dev.put(x)
    stream = torch.cuda.Stream()
    for call in range(2):
        d_out = dev.empty(x.nbytes)
        st = lib.parallax_scan_noalloc(h, d_in.data_ptr(), d_out.data_ptr(), n, s,
                                       init.ctypes.data if exclusive else None,
                                       C.c_void_p(stream.cuda_stream))
        assert st == px.OK, (call, st)
        got = dev.get(d_out, x.dtype, n)
        if t in ("f32", "f64"):
            want_f = ox.scan(x, exclusive=exclusive, init=3 if exclusive else 0)
            assert same(t, got, want_f), call
            assert same(t, got.astype(np.float64), want.astype(np.float64)), call
        else:
            assert np.array_equal(got, want), call


def test_noalloc_in_place(lib, px, ox, dev):
    x = gen(ox, "i32", 100003, seed=42)
    d = dev.put(x)
    h = px.builtin("scan:i32")
    assert lib.parallax_scan_noalloc(h, d.data_ptr(), d.data_ptr(), x.size, 4, None, None) == px.OK
    assert np.array_equal(dev.get(d, np.int32, x.size), ox.scan(x))


def test_noalloc_rejects_counts_beyond_its_static_capacity(lib, px, dev):
    h = px.builtin("scan:u32")
    d = dev.empty(64)
    too_many = MAX_TILES * TILE[4] + 1
    st = lib.parallax_scan_noalloc(h, d.data_ptr(), d.data_ptr(), too_many, 4, None, None)
    assert st == px.ERR_INVALID_ARGUMENT
    assert lib.parallax_last_error() == px.ERR_INVALID_ARGUMENT
    lib.parallax_clear_error()
    h8 = px.builtin("scan:i64")
    st = lib.parallax_scan_noalloc(h8, d.data_ptr(), d.data_ptr(), MAX_TILES * TILE[8] + 1, 8,
                                   None, None)
    assert st == px.ERR_INVALID_ARGUMENT
    lib.parallax_clear_error()


def test_noalloc_largest_count(lib, px, ox, dev):
    torch = dev.torch
    n = MAX_TILES * TILE[8]
    d = torch.ones(n, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    h = px.builtin("scan:i64")
    assert lib.parallax_scan_noalloc(h, d.data_ptr(), d.data_ptr(), n, 8, None, None) == px.OK
    idx = np.unique(np.concatenate([[0, 1, n - 2, n - 1], np.arange(0, n, 4099)]))
    got = d[torch.from_numpy(idx).cuda()].cpu().numpy()
    assert np.array_equal(got, idx + 1)
    del d
